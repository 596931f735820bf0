"""CPU oracle for the photoemission tracer's hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path (``bem_b200``) never
imports anything from here and fails loudly when its CUDA library is
missing.

It is a plain NumPy/SciPy restatement, in float64, of the reference
package ``specific_particle_tracer`` (AdamCBartnik/BEM) for exactly the
functions on the hot path:

* ``physics``  -- constants, Plummer pair sums, flat and 3-image image
  forces, analytic gun / hemispherical-tip fields, kill masks
  (``forces.py``, ``fields.py``, ``geometry.py``, ``constants.py``);
* ``bem``      -- ring field with K(1-p), E(1-p), fixed far quadrature,
  closest point, near-segment sinh quadrature, blend with the flat
  fallback (``bem/axisymmetric.py``, ``bem/_elliptic.py``,
  ``bem/fields.py``, ``bem/geometry.py``);
* ``rk45``     -- the per-group adaptive Dormand-Prince 5(4) driver with
  birth checkpoints, output-time landing, kill-after-accept and the RMS
  error norm (``batched_rk45.py``), instrumented with a per-group attempt
  log (h, error norm, accepted) for acceptance-sequence parity;
* ``screens``  -- Hermite screen-crossing detection (``screens.py``);
* ``geometry`` -- builds accel/kill callables from a plain geometry spec.

Parity is pinned: ``tests/test_oracle_golden.py`` checks every function
here against fixtures produced by running the reference itself
(``tests/golden/make_golden.py``), which imports the reference package
from its source tree in the development container.
"""
