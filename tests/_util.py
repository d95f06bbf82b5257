import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def t2n(t):
    """torch tensor in the (3,npoin)/(64,nelem) storage -> numpy in the reference Fortran shape."""
    a = t.detach().cpu().numpy()
    return np.asfortranarray(a.T) if a.ndim == 2 else a
