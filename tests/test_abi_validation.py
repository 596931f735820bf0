"""Argument checks of the C ABI, which run on the host before any device
work: bad inputs come back as error codes with a message, never as a launch.
Each call here returns before its first CUDA call, so no GPU is needed."""

import ctypes

import pytest

from bem_b200 import _lib

torch = pytest.importorskip("torch")
# The structs below carry made-up device addresses.  Every case returns
# before a launch, but should a check ever let one through, a GPU would be
# given those addresses: these host-logic tests run only where no GPU is.
pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="host-only checks with made-up device addresses")

FAKE = 1 << 20  # a 256-byte aligned address that is never dereferenced on these paths


def _state(n_groups=1, max_size=32):
    s = _lib.SptState()
    s.n_groups = n_groups
    s.max_group_size = max_size
    return s


def _params(form=_lib.FORM_FP64):
    p = _lib.SptTraceParams()
    p.form = form
    return p


def _geom(kind=_lib.GEOM_FLAT):
    g = _lib.SptGeometry()
    g.kind = kind
    return g


def _bem(**kw):
    b = _lib.SptBem()
    b.n_seg, b.nodes_per_seg, b.seg_stride, b.node_stride = 10, 32, 10, 320
    b.seg, b.node = FAKE, FAKE
    for k, v in kw.items():
        setattr(b, k, v)
    return b


def _trace(state, params, geom, bem=None):
    L = _lib.lib()
    return L.spt_trace(ctypes.byref(state), ctypes.byref(params), ctypes.byref(geom),
                       ctypes.byref(bem) if bem is not None else None, ctypes.c_void_p(FAKE), 1 << 20, None)


def test_empty_batch_is_a_no_op():
    assert _trace(_state(n_groups=0), _params(), _geom()) == _lib.SPT_OK


def test_group_size_beyond_the_maximum():
    assert _trace(_state(max_size=1025), _params(), _geom()) == _lib.SPT_ERR_CAPACITY
    assert "max_group_size" in _lib.last_error()


def test_active_count_needs_an_order():
    s = _state()
    s.n_active = FAKE
    assert _trace(s, _params(), _geom()) == _lib.SPT_ERR_ARG
    assert "n_active needs group_order" in _lib.last_error()


def test_unknown_form():
    assert _trace(_state(), _params(form=7), _geom()) == _lib.SPT_ERR_ARG
    assert "unknown form" in _lib.last_error()


def test_bem_geometry_needs_tables():
    assert _trace(_state(), _params(), _geom(_lib.GEOM_POST_BEM)) == _lib.SPT_ERR_ARG
    assert "BEM tables required" in _lib.last_error()


@pytest.mark.parametrize("kw,msg", [
    (dict(far_rule=5), "unknown far rule"),
    (dict(far_rule=_lib.FAR_ADAPTIVE), "coarse node table"),
    (dict(far_rule=_lib.FAR_ADAPTIVE, coarse=FAKE, coarse_stride=60, ratio4=0.5, ratio2=300.0), "ratio4"),
    (dict(far_rule=_lib.FAR_ADAPTIVE, coarse=FAKE, coarse_stride=60, ratio4=8.0, ratio2=4.0), "ratio4 <= ratio2"),
    (dict(far_rule=_lib.FAR_ADAPTIVE, coarse=FAKE, coarse_stride=60, ratio4=8.0, ratio2=300.0, blk=FAKE,
          blk_stride=1, run_nodes=FAKE, run_stride=4, ratio_run=4.0), "run-node table too small"),
    (dict(far_rule=_lib.FAR_ADAPTIVE, coarse=FAKE, coarse_stride=60, ratio4=8.0, ratio2=300.0, blk=FAKE,
          blk_stride=1, run_nodes=FAKE, run_stride=8, ratio_run=0.5), "ratio_run"),
    (dict(nodes_per_seg=30), "multiple of 4"),
])
def test_bem_table_checks(kw, msg):
    rc = _trace(_state(), _params(), _geom(_lib.GEOM_POST_BEM), _bem(**kw))
    assert rc == _lib.SPT_ERR_ARG
    assert msg in _lib.last_error()


def test_learned_form_needs_its_parameters():
    rc = _trace(_state(), _params(form=_lib.FORM_SURROGATE), _geom(_lib.GEOM_POST_BEM), _bem())
    assert rc == _lib.SPT_ERR_ARG
    assert "surrogate parameters missing" in _lib.last_error()


def test_other_entry_points_reject_null_arguments():
    L = _lib.lib()
    assert L.spt_compact_groups(None, 4, None, None, None, None) == _lib.SPT_ERR_ARG
    assert L.spt_bem_field(None, None, None, 0, None, 0, None, None, None, None) == _lib.SPT_OK  # n = 0
    rc = L.spt_surrogate_field(FAKE, FAKE, FAKE, 4, ctypes.byref(_bem()), None, FAKE, FAKE, FAKE, None)
    assert rc == _lib.SPT_ERR_ARG


def test_unknown_team():
    p = _params()
    p.team = 7
    assert _trace(_state(), p, _geom()) == _lib.SPT_ERR_ARG
    assert "unknown team" in _lib.last_error()


@pytest.mark.parametrize("form,kind,size", [(_lib.FORM_FP64, _lib.GEOM_FLAT, 32),
                                            (_lib.FORM_MIXED, _lib.GEOM_FLAT, 32)])
def test_warp_team_where_not_offered(form, kind, size):
    """One group per warp serves BEM geometries in the float64 form with the
    adaptive far rule and groups of at most 32 particles; asked for anywhere
    else, the call fails before any device work."""
    p = _params(form)
    p.team = _lib.TEAM_WARP
    assert _trace(_state(max_size=size), p, _geom(kind)) == _lib.SPT_ERR_ARG
    assert "warp team needs" in _lib.last_error()


def _workspace(state, params, geom, bem):
    n = ctypes.c_int64(0)
    rc = _lib.lib().spt_trace_workspace_bytes(ctypes.byref(state), ctypes.byref(params), ctypes.byref(geom),
                                              ctypes.byref(bem), ctypes.byref(n))
    assert rc == _lib.SPT_OK
    return n.value


def test_workspace_holds_the_warp_teams_slots():
    """Groups of at most 32 in the float64 form with the adaptive rule: the
    workspace holds one step slot (54 doubles a particle, 32 lanes) per warp
    of the warp team's grid -- without a device, SMs x two 256-thread CTAs,
    no more than the groups need; one group per CTA needs only the queue
    counter."""
    geom = _geom(_lib.GEOM_POST_BEM)
    bem = _bem(far_rule=_lib.FAR_ADAPTIVE)
    slot = 54 * 32 * 8
    p = _params()
    n = _workspace(_state(n_groups=4096, max_size=32), p, geom, bem)
    assert n == 256 + 148 * 2 * 8 * slot
    assert _workspace(_state(n_groups=20, max_size=32), p, geom, bem) == 256 + 3 * 8 * slot
    p.team = _lib.TEAM_CTA
    assert _workspace(_state(n_groups=4096, max_size=32), p, geom, bem) == 256
    p.team = _lib.TEAM_AUTO
    assert _workspace(_state(n_groups=4096, max_size=33), p, geom, bem) == 256
    assert _workspace(_state(n_groups=4096, max_size=32), _params(_lib.FORM_MIXED), geom, bem) == 256
