"""The host side of the mode-split step (adaptive.py:ModeSplitOcean.step) on
CPU, against a fake device handle that records its calls: the order of the
device calls in one step, and time_step's remap test (src/main.f90:447-454):
the layers are remapped exactly when the smallest relative layer mass is below
min_mass_remap, with the hybrid coefficients of the initial layers."""
import numpy as np

from wavetrisk_hydrostatic_b200.adaptive import ModeSplitOcean


class _Report:
    status = 0


class _FakeDev:
    def __init__(self, masses):
        self.masses = list(masses)
        self.calls = []

    def rk4_split(self, dt, theta1, theta2, solver):
        self.calls.append("rk4_split")
        return _Report()

    def adapt(self, threshold, level_fill, max_level):
        self.calls.append("adapt")

    def inverse_tree(self):
        self.calls.append("inverse_tree")

    def inverse(self):
        self.calls.append("inverse")

    def mask_build(self, *a):
        self.calls.append("mask_build")

    def compress(self):
        self.calls.append("compress")

    def free_surface_adapt(self):
        self.calls.append("free_surface_adapt")

    def min_mass(self, b_vert):
        self.calls.append("min_mass")
        self.b_seen = np.array(b_vert)
        return self.masses.pop(0)

    def remap_vertical(self, kind, a_vert, b_vert):
        self.calls.append(("remap", kind))
        self.ab_seen = (np.array(a_vert), np.array(b_vert))


def _model(masses, remap="2PPM", tree=True, nz=4):
    m = object.__new__(ModeSplitOcean)   # the host logic only: no device, no grid
    m.dev = _FakeDev(masses)
    m.dt, m.theta1, m.theta2, m.solver = 600.0, 1.0, 1.0, None
    m.tree, m.dynamic, m.istep = tree, False, 0
    m.threshold_def = np.ones((3, nz))
    m.threshold = m.threshold_def.copy()
    m.level_fill, m.max_level = 0, 5
    m.remap, m.min_mass_remap, m.remaps = remap, 0.9, 0
    m.b_vert = 1.0 - np.arange(nz + 1) / nz
    m.a_vert = 1.0 - m.b_vert
    m.min_mass = None
    return m


def test_step_order_on_a_tree():
    m = _model([0.95])
    m.step()
    assert m.dev.calls == ["rk4_split", "adapt", "inverse_tree", "free_surface_adapt", "min_mass"]
    assert m.remaps == 0 and m.min_mass == 0.95 and m.istep == 1


def test_remap_exactly_below_min_mass_remap():
    m = _model([0.95, 0.9, 0.899, 0.5, 0.0])
    for _ in range(5):
        m.step()
    remaps = [c for c in m.dev.calls if isinstance(c, tuple)]
    assert remaps == [("remap", "2PPM")] * 3 and m.remaps == 3      # 0.899, 0.5 and a collapsed layer
    a, b = m.dev.ab_seen
    assert np.array_equal(b, [1.0, 0.75, 0.5, 0.25, 0.0]) and np.array_equal(a + b, np.ones(5))
    assert np.array_equal(m.dev.b_seen, b)


def test_no_remap_test_when_off_and_dense_path():
    m = _model([], remap=None, tree=False)
    m.step()
    assert m.dev.calls == ["rk4_split", "mask_build", "compress", "inverse", "free_surface_adapt"]
    assert m.remaps == 0 and m.min_mass is None
