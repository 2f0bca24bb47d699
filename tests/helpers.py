"""Shared helpers for the parity tests: seeded inputs, boundary-condition sets, oracle access."""
import numpy as np

from oracle import oracle_ctypes as O

F32, F64 = O.F32, O.F64
NEU, DIR, PER, NONE, INFLOW = 4, 3, 2, 1, 7


def npdt(dt):
    return np.float64 if dt == F64 else np.float32


def rand_buffer(L, dt, rng, lo=-1.0, hi=1.0):
    """Random values in every element of a padded buffer (ghosts and padding included)."""
    return rng.uniform(lo, hi, int(L.allocated)).astype(npdt(dt))


def bc_from(spec):
    """spec: dict face -> (type, value[, aux]) or a single (type, value) for all faces."""
    if isinstance(spec, tuple):
        return O.bcset_all(*spec)
    return O.bcset(**spec)


SCALAR_BCS = {
    "neumann": (NEU, 0.0),
    "neumann_inhom": {"xpos": (NEU, 0.25), "xneg": (NEU, -0.5), "ypos": (NEU, 1.0), "yneg": (NEU, 0.0),
                      "zpos": (NEU, -0.75), "zneg": (NEU, 0.125)},
    "dirichlet": (DIR, 0.321),
    "periodic": (PER, 0.0),
    "mixed_xdir": {"xpos": (DIR, 1.0), "xneg": (DIR, 1.0), "ypos": (PER, 0), "yneg": (PER, 0),
                   "zpos": (PER, 0), "zneg": (PER, 0)},
    "mixed_zneu": {"xpos": (PER, 0), "xneg": (PER, 0), "ypos": (PER, 0), "yneg": (PER, 0),
                   "zpos": (NEU, 0.0), "zneg": (NEU, 0.0)},
    "mixed_all": {"xpos": (DIR, -1.0), "xneg": (NEU, 0.5), "ypos": (PER, 0), "yneg": (PER, 0),
                  "zpos": (NONE, 0), "zneg": (DIR, 0.25)},
    "mixed_dn": {"xpos": (DIR, 0.5), "xneg": (NEU, -0.25), "ypos": (NEU, 0.75), "yneg": (DIR, -0.125),
                 "zpos": (DIR, 1.5), "zneg": (NEU, 0.375)},
}

MAC_BCS = {
    "closed_noslip": (INFLOW, 0.0, 1.0),
    "closed_freeslip": (INFLOW, 0.0, 0.0),
    "periodic": (PER, 0.0),
    "rb": {"xpos": (PER, 0), "xneg": (PER, 0), "ypos": (PER, 0), "yneg": (PER, 0),
           "zpos": (INFLOW, 0.0, 1.0), "zneg": (INFLOW, 0.0, 1.0)},
    "inflow": {"xpos": (INFLOW, 0.5, 0.0), "xneg": (INFLOW, 0.5, 0.0), "ypos": (PER, 0), "yneg": (PER, 0),
               "zpos": (INFLOW, 0.0, 1.0), "zneg": (INFLOW, 0.0, 0.5)},
}


def mg_params(bc, nu1=2, nu2=2, conv=0x05, sym=0, disable_host=0):
    p = O.MGParams()
    p.bc = bc
    p.nu1, p.nu2, p.convergence = nu1, nu2, conv
    p.make_symmetric_operator = sym
    p.disable_relax_on_host = disable_host
    return p


def config1_rhs(n=64, seed=0):
    """64^3 FP32 pressure config: RHS ~ U[-1,1] i.i.d. from the seed, FP64 mean subtracted."""
    rng = np.random.default_rng(seed)
    b = rng.uniform(-1.0, 1.0, (n, n, n))
    b -= b.mean()
    return b
