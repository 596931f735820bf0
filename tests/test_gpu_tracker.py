"""Tracker-level parity: bem_b200.SpecificParticleTracer(backend='b200') against
the reference's own SpecificParticleTracer run (screens + t_out) recorded in
tests/golden/tracker_flat.npz."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from bem_b200 import SpecificParticleTracer, workloads  # noqa: E402
from bem_b200 import geometry as bg  # noqa: E402


class _Particles:
    """The ParticleGroup attributes the tracker reads (tracker.py:214-284)."""

    def __init__(self, d):
        for k, v in d.items():
            setattr(self, k, v)
        self.mass = 510998.95069
        self.species_charge = -1.602176634e-19
        self.species = "electron"

    def __len__(self):
        return len(self.x)


KEYS = ("x", "y", "z", "px", "py", "pz", "t")


def _sorted(ids, t, cols):
    o = np.lexsort((t, ids))
    return ids[o], [c[o] for c in cols]


def test_tracker_screens_and_outputs_match_reference():
    g = load_golden("tracker_flat")
    d = workloads.flat_c0(n_groups=3, n_emit=6, seed=31)
    pg = _Particles({k: v for k, v in d.items() if k != "group_sizes"})
    tr = SpecificParticleTracer(pg, 6, bg.FlatCathode(-1e7), screens=[1e-7, 5e-6], t_out=[0.5e-12, 1.5e-12],
                                rtol=1e-8, z_max=2e-5)
    assert tr.t_max == pytest.approx(float(g["t_max"]), rel=1e-15)
    screens, trajs = tr.run()
    for k, s in enumerate(screens):
        ref_ids = g[f"screen{k}_id"]
        assert len(s) == len(ref_ids)
        if len(ref_ids) == 0:
            continue
        ids, mine = _sorted(np.asarray(s.id), np.asarray(s.t), [np.asarray(getattr(s, c)) for c in KEYS])
        rids, ref = _sorted(ref_ids, g[f"screen{k}_t"], [g[f"screen{k}_{c}"] for c in KEYS])
        np.testing.assert_array_equal(ids, rids)
        for a, b, c in zip(mine, ref, KEYS):
            np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6 * np.abs(b).max(), err_msg=f"screen {k} {c}")
    for k, s in enumerate(trajs):
        ref_ids = g[f"traj{k}_id"]
        assert len(s) == len(ref_ids)
        ids, mine = _sorted(np.asarray(s.id), np.asarray(s.t), [np.asarray(getattr(s, c)) for c in KEYS])
        rids, ref = _sorted(ref_ids, g[f"traj{k}_t"], [g[f"traj{k}_{c}"] for c in KEYS])
        np.testing.assert_array_equal(ids, rids)
        for a, b, c in zip(mine, ref, KEYS):
            np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6 * np.abs(b).max(), err_msg=f"t_out {k} {c}")


def test_tracker_rejects_workers_and_bad_grouping():
    d = workloads.flat_c0(n_groups=2, n_emit=4, seed=3)
    pg = _Particles({k: v for k, v in d.items() if k != "group_sizes"})
    with pytest.raises(ValueError):
        SpecificParticleTracer(pg, 4, bg.FlatCathode(-1e7), screens=[], n_workers=2)
    with pytest.raises(ValueError):
        SpecificParticleTracer(pg, 3, bg.FlatCathode(-1e7), screens=[])
