"""Minimal stand-in for openpmd-beamphysics' ParticleGroup, used only when
tests/golden/make_golden.py imports the reference package to produce
fixtures.  It stores the data dict, exposes it as attributes and gives the
electron rest mass and charge the reference reads (tracker.py:219-229)."""

import numpy as np

_E = 1.602176634e-19


class ParticleGroup:
    def __init__(self, data=None, **kw):
        data = dict(data or {}, **kw)
        self._data = {k: (np.asarray(v) if k != "species" else v) for k, v in data.items()}
        self.species = data.get("species", "electron")
        self.mass = 510998.95069
        self.species_charge = -_E

    def __getattr__(self, name):
        d = self.__dict__.get("_data", {})
        if name in d:
            return d[name]
        raise AttributeError(name)

    def __len__(self):
        return len(self._data["x"])
