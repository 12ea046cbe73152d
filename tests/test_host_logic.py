"""Host logic without a GPU: the launch-shape autotuner's coordinate
descent, snapshot/restore and JSON cache on a fake run whose stage times
are a known function of the shapes; the film's conversion of the device
counts into the script's charges."""
import json
import types

import numpy as np

from conftest import load_package

vb = load_package()
AT = vb.autotune


class FakeAccelerator:
    """Stage times as a function of the launch shapes: the forces stage is
    fastest with the tensor-core gather and chunk 128, the coarse deposit
    with 4 CTAs per SM, the push with 2; the others do not matter."""

    def __init__(self):
        self.shapes = {"field_tensor_cores": 0, "chunk": 64, "field_ctas_per_sm": 3, "cic_ctas_per_sm": 2,
                       "push_ctas_per_sm": 4, "move_ctas_per_sm": 8}
        self.profiling = False
        self.acc_ms = {}
        self.device = 0

    def tuning(self):
        return dict(self.shapes)

    def set_tuning(self, **kw):
        assert set(kw) <= set(self.shapes)
        self.shapes.update(kw)

    def profile(self, on):
        self.profiling = on
        if on:
            self.acc_ms = {}

    def record_step(self):
        s = self.shapes
        t = {
            "sort": 0.43 + (0.01 if s["chunk"] == 256 else 0.0) + 0.001 * abs(s["move_ctas_per_sm"] - 8),
            "deposit_coarse": 0.19 + 0.02 * abs(s["cic_ctas_per_sm"] - 4) + 0.01 * (s["chunk"] != 128),
            "forces": (0.95 if s["field_tensor_cores"] else 1.04) + 0.05 * (s["chunk"] != 128),
            "push": 0.17 + 0.001 * s["push_ctas_per_sm"],
        }
        if self.profiling:
            for k, v in t.items():
                self.acc_ms[k] = self.acc_ms.get(k, 0.0) + v

    def stage_times(self):
        return dict(self.acc_ms)


class FakeSim:
    def __init__(self):
        self.accelerator = FakeAccelerator()
        self.use_graph = True
        self.state = 0               # stands for the cloud and the projectile
        self.meshes = types.SimpleNamespace(fine=types.SimpleNamespace(n=130))
        self.params = types.SimpleNamespace(nparticles=8_000_000)

    def step(self):
        assert self.use_graph is False or not self.accelerator.profiling
        self.state += 1
        self.accelerator.record_step()

    def snapshot(self):
        return self.state

    def restore(self, snap):
        self.state = snap


def test_autotune_descends_each_coordinate_and_restores_the_run():
    sim = FakeSim()
    sim.state = 41
    best = AT.tune(sim, steps=2, warmup=1)
    assert best["field_tensor_cores"] == 1
    assert best["chunk"] == 128
    assert best["cic_ctas_per_sm"] == 4
    assert best["push_ctas_per_sm"] == 2
    assert sim.accelerator.tuning() == best       # left set on the run
    assert sim.state == 41 and sim.use_graph       # the run as it was
    assert not sim.accelerator.profiling


def test_autotune_cache_round_trip(tmp_path):
    path = tmp_path / "tuning.json"
    sim = FakeSim()
    best = AT.tune_cached(sim, path, steps=1, warmup=0)
    cache = json.loads(path.read_text())
    assert list(cache.values()) == [best]
    # a second run of the same kind takes the cached shapes without stepping
    other = FakeSim()
    other.step = None
    assert AT.tune_cached(other, path) == best
    assert other.accelerator.tuning() == best


def test_film_counts_become_the_scripts_charges():
    frames = np.arange(2 * 4 * 4, dtype=np.float32).reshape(2, 4, 4)
    scalars = np.array([[-20.0, 10.0, 30.0, 100.0], [-19.8, 10.0, 40.0, 90.0]])
    acc = types.SimpleNamespace(film_download=lambda: (frames, scalars), film_frames=lambda: (3, 2))
    fake = types.SimpleNamespace(accelerator=acc, weight=196.0 / 1000, jellium=vb.Jellium.of(196.0))
    f = vb.Simulation.film_frames(fake)
    assert f.taken == 3 and f.frames is frames
    assert np.array_equal(f.proj_x, [-20.0, -19.8]) and np.array_equal(f.proj_y, [10.0, 10.0])
    assert np.allclose(f.q_capture, [30 * 0.196, 40 * 0.196], rtol=0, atol=1e-12)
    assert np.allclose(f.q_net, [196 - 100 * 0.196, 196 - 90 * 0.196], rtol=0, atol=1e-12)
