"""Load the golden fixtures written by tests/golden/make_golden.py."""
import os

import numpy as np
import scipy.sparse as sp

from orbit_b200 import synthetic

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_grid.npz")
_NAMES = ("dP", "Dz", "u", "v", "u_plus", "u_minus", "v_plus", "v_minus", "u_e",
          "u_plus_e", "u_minus_e", "v_n", "v_plus_n", "v_minus_n", "kxxyy", "kzz",
          "w_plus", "w_minus", "cmfmc", "kmu", "kmv", "lat", "lon")


PRESSURE_FORM = os.path.join(os.path.dirname(GOLDEN), "pressure_form.npz")


def load():
    return dict(np.load(GOLDEN))


def load_pressure_form():
    """Goldens of a grid in the pressure form (concentration_state False) and its MetBin."""
    z = dict(np.load(PRESSURE_FORM))
    m = met_bin(z, "pf_")
    m.concentration_state = False
    return z, m


def met_bin(z, prefix):
    nz, ny, nx, dlat, dlon, split = z[f"{prefix}meta"]
    kw = {n: np.array(z[f"{prefix}{n}"]) for n in _NAMES}
    if f"{prefix}u_wrap" in z:
        kw["periodic_lon"] = True
        for n in ("u_wrap", "u_plus_wrap", "u_minus_wrap", "kmu_wrap"):
            kw[n] = np.array(z[f"{prefix}{n}"])
    return synthetic.MetBin(nz=int(nz), ny=int(ny), nx=int(nx), dlat=float(dlat),
                            dlon=float(dlon), split=bool(split), **kw)


PERIODIC = os.path.join(os.path.dirname(GOLDEN), "periodic.npz")


def load_periodic():
    """Goldens of periodic-longitude grids (tests/golden/make_golden.py --periodic)."""
    return dict(np.load(PERIODIC))


def met_list(z):
    return [met_bin(z, f"met{t}_") for t in range(8)]


def species(z):
    return synthetic.SpeciesFields(vd=z["vd"], wet=z["wet"], loss=z["loss"], emis=z["emis"])


def csc(z, prefix):
    n = len(z[f"{prefix}indptr"]) - 1
    return sp.csc_matrix((z[f"{prefix}data"], z[f"{prefix}indices"], z[f"{prefix}indptr"]),
                         shape=(n, n))
