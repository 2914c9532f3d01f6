"""Physical constants used on the integral path (PyQuante/Constants.py:20-21)."""
bohr2ang = 0.529177249   # bohr -> angstrom
ang2bohr = 1 / bohr2ang
hartree2kcal = 627.5095
