"""The C ABI without a GPU: the library loads, exports every symbol the
header declares, and turns bad arguments into status codes (the reference's
argument errors, src/accelerator.jl:262-268, 583-586, become VLB_ERR_ARG)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from conftest import ROOT, load_package

vb = load_package()
L = vb._lib


def header_symbols():
    text = (ROOT / "include" / "vlasov_b200.h").read_text()
    return sorted(set(re.findall(r"^VLB_API\s+[\w\s\*]+?\b(vlb_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(built):
    lib = C.CDLL(str(L.LIB_PATH))
    declared = header_symbols()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(L.EXPORTS) == declared
    assert b"sm_100a" in L.lib().vlb_version()


def test_null_and_bad_arguments_return_codes(built):
    lib = L.lib()
    assert lib.vlb_destroy(None) == L.VLB_ERR_ARG
    assert lib.vlb_create(None, None) == L.VLB_ERR_ARG
    assert b"null" in lib.vlb_last_error()
    assert lib.vlb_sort(None, None, None) == L.VLB_ERR_ARG
    assert lib.vlb_step(None, None, None, None) == L.VLB_ERR_ARG


def _config(vb, nfine=16, npart=100, nonuniform=False):
    m = vb.build_meshes(nfine, *vb.grids(nfine), 78.0, 235.0)
    if nonuniform:
        m.fine.axis.knots = m.fine.axis.knots.copy()
        m.fine.axis.knots[2] += 0.3
    sm = vb.gaussian_smoothing(m.fine.axis, nbdt=50, quadrature=50)
    keep = []
    cfg = L.Config()
    cfg.npart, cfg.weight = npart, 196 / max(npart, 1)
    from vlasov_b200.simulation import _level_desc
    cfg.fine = _level_desc(m.fine, keep)
    cfg.coarse = _level_desc(m.coarse, keep)
    s = L.SmoothingDesc()
    s.nbdt, s.spacing = sm.nbdt, sm.spacing
    for name, tab in (("overlap", sm.overlap), ("gradient", sm.gradient), ("nodes", sm.nodes)):
        a = np.ascontiguousarray(tab.T)
        keep.append(a)
        setattr(s, name, L.pd(a))
    cfg.smoothing = s
    return cfg, keep


def test_create_rejects_bad_configs_before_touching_a_device(built):
    lib = L.lib()
    h = C.c_void_p()
    cfg, keep = _config(vb, npart=0)
    assert lib.vlb_create(C.byref(cfg), C.byref(h)) == L.VLB_ERR_ARG
    assert b"npart" in lib.vlb_last_error()
    cfg, keep = _config(vb, nonuniform=True)
    assert lib.vlb_create(C.byref(cfg), C.byref(h)) == L.VLB_ERR_ARG
    assert b"uniform" in lib.vlb_last_error()
    cfg, keep = _config(vb)
    cfg.weight = -1.0
    assert lib.vlb_create(C.byref(cfg), C.byref(h)) == L.VLB_ERR_ARG
    cfg, keep = _config(vb)
    cfg.smoothing.overlap = None
    assert lib.vlb_create(C.byref(cfg), C.byref(h)) == L.VLB_ERR_ARG
    assert not h.value


def test_host_helpers_round_trip(built):
    rng = np.random.default_rng(5)
    pos = rng.uniform(-200, 200, (1000, 3))
    k, d = vb.pack_positions(pos, -78.0, 2.4375)
    back = vb.unpack_positions(k, d, -78.0, 2.4375)
    assert np.max(np.abs(back - pos)) < 1e-6
    assert np.all(np.abs(d) <= 2.4375 / 2 + 1e-6)
    assert k.min() < 1 and k.max() > 65   # unclamped (src/particles.jl:58-61)
