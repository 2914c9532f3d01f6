"""6-31G* basis: 6-31G** with the p polarisation shell removed from H and He
(the d shells on heavier atoms stay).  Derived from p631ss at import."""
from .p631ss import basis_data as _p631ss

basis_data = {z: [(sym, prims) for (sym, prims) in shells if not (z <= 2 and sym == "P")]
              for z, shells in _p631ss.items()}
