"""Module-level state of the drop-in API, with the names and layouts of the
reference's python/shared.py:15-66 (set by ``read_input``):

  M, ne, nst, svh, skp, siv, efs
  mass (ne, ne), ncv (ne+1,), scvv (nst,) already divided by nst,
  sml (ne, ne, nst), sms (skp, skp, nst), iv (siv,), C (M,),
  H, S, Kinetic, Potential (M, M), grad (siv + M,)

The dense per-pair derivative matrices DH/DS of the reference are never
materialised: the gradient kernels contract them with C on the fly.
``sync_matrices`` controls whether outprod copies H and S back into this
module after each call, as the reference's outprod does as a side effect.
"""
import math

import numpy as np

M: int = 0
ne: int = 0
NN: int = 0
nst: int = 0
svh: int = 0
skp: int = 0
siv: int = 0
efs: float = 0.0
mass: np.ndarray = None
S: np.ndarray = None
H: np.ndarray = None
Kinetic: np.ndarray = None
Potential: np.ndarray = None
grad: np.ndarray = None
GRADA: np.ndarray = None
GRADC: np.ndarray = None
iv: np.ndarray = None
ncv: np.ndarray = None
scvv: np.ndarray = None
C: np.ndarray = None
sml: np.ndarray = None
sms: np.ndarray = None
PI: float = math.pi
sync_matrices: bool = True
