"""Host logic of the autotuner's team knob (no GPU): which tracers and group
sizes the warp team is offered for -- the predicate of the C ABI's team
selection -- and how a tuned configuration is applied to a tracer."""

from types import SimpleNamespace

import numpy as np
import pytest

from bem_b200 import _lib, autotune


def _tracer(form=_lib.FORM_FP64, far_rule="adaptive", kind=_lib.GEOM_POST_BEM, has_image=1, image_nodes=0,
            tables=True):
    bem = SimpleNamespace(image=SimpleNamespace(n_nodes=image_nodes))
    return SimpleNamespace(form=form, far_rule=far_rule, tables=object() if tables else None,
                           bem=bem if tables else None, geom=SimpleNamespace(kind=kind, has_image=has_image),
                           round_points=0, cta_threads=0, team=_lib.TEAM_AUTO)


@pytest.mark.parametrize("kw,sizes,offered", [
    ({}, [32, 1, 7], True),                                    # C1 / C4 small bins: float64, adaptive, <= 32
    ({}, [33], False),                                         # a group above one warp
    (dict(form=_lib.FORM_MIXED), [32], False),                 # the float32 form
    (dict(far_rule="reference"), [32], False),                 # the plain form's quadrature
    (dict(tables=False, kind=_lib.GEOM_FLAT), [32], False),    # no BEM field
    (dict(kind=_lib.GEOM_TIP_BEM, image_nodes=53), [8], False),  # the BEM image-charge force (a CTA routine)
    (dict(kind=_lib.GEOM_TIP_BEM, image_nodes=0), [8], True),  # a BEM tip without image tables
    (dict(kind=_lib.GEOM_WELL_BEM, has_image=0, image_nodes=0), [16], True),
])
def test_warp_team_offered(kw, sizes, offered):
    assert autotune.warp_team_offered(_tracer(**kw), np.asarray(sizes)) is offered


def test_apply_maps_the_tuned_team():
    cfg = dict(team=_lib.TEAM_WARP, cta_threads=128, round_points=2, ratios=[8.0, 300.0, 4.0],
               order="largest_first")
    tr = _tracer(tables=False)
    autotune.apply(cfg, tr)
    # the warp team becomes the library's choice: it takes the launches whose groups fill the GPU
    assert (tr.team, tr.cta_threads, tr.round_points) == (_lib.TEAM_AUTO, 128, 2)
    autotune.apply(dict(cfg, team=_lib.TEAM_CTA), tr)
    assert tr.team == _lib.TEAM_CTA
    autotune.apply({k: v for k, v in cfg.items() if k != "team"}, tr)
    assert tr.team == _lib.TEAM_AUTO
