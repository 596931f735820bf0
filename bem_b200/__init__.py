"""bem_b200 -- B200-native (sm_100a) backend for the specific_particle_tracer
hot path: the adaptive per-group Dormand-Prince RK45 photoemission tracer with
in-group Coulomb/image pair forces and an axisymmetric BEM ring-charge field.

Importing the package loads nothing on the GPU; the CUDA library is loaded on
first use (and its absence is an error, never a fallback)."""

__all__ = ["SpecificParticleTracer", "FlatCathode", "HemisphericalTip", "HemisphericalTipBEMGeometry",
           "CylindricalWellBEMGeometry", "PostTipBEMGeometry", "from_reference", "resolve_backend"]


def __getattr__(name):
    if name == "SpecificParticleTracer":
        from .tracker import SpecificParticleTracer
        return SpecificParticleTracer
    if name == "resolve_backend":
        from .backend import resolve_backend
        return resolve_backend
    if name in ("FlatCathode", "HemisphericalTip", "HemisphericalTipBEMGeometry", "CylindricalWellBEMGeometry",
                "PostTipBEMGeometry", "from_reference"):
        from . import geometry
        return getattr(geometry, name)
    raise AttributeError(name)
