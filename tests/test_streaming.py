"""The seeded cloud drawn as a stream (vlb_sampler; the construction of
src/initial.jl:94-113 a chunk at a time), without a GPU: consecutive draws
of any sizes give the one-shot cloud bit for bit, and skipped particles
consume the generator as drawn ones do (a rank keeping only its slice)."""
import numpy as np

from conftest import load_package

vb = load_package()


def test_chunked_draws_are_the_one_shot_cloud(built):
    prof = vb.thomas_fermi_profile()
    n, w = 50_000, 196 / 50_000
    pos, mom = vb.sample_thomas_fermi(prof, n, w, seed=-3)
    st = vb.ThomasFermiStream(prof, w, seed=-3)
    parts, got = [], 0
    for size in (1, 4095, 4096, 1 << 14, 7):
        parts.append(st.draw(size))
        got += size
    parts.append(st.draw(n - got))
    st.close()
    p2 = np.concatenate([p for p, _ in parts])
    m2 = np.concatenate([m for _, m in parts])
    assert np.array_equal(pos, p2) and np.array_equal(mom, m2)


def test_skipped_particles_consume_the_stream(built):
    prof = vb.uniform_sphere_profile()
    n, w = 30_000, 196 / 30_000
    pos, mom = vb.sample_thomas_fermi(prof, n, w, seed=-1)
    for lo, hi in ((0, 10_000), (10_000, 20_001), (20_001, 30_000)):
        st = vb.ThomasFermiStream(prof, w, seed=-1)
        st.skip(lo)
        p, m = st.draw(hi - lo)
        st.close()
        assert np.array_equal(p, pos[lo:hi]) and np.array_equal(m, mom[lo:hi])
