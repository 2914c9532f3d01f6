"""Basis-set name lookup (PyQuante/Basis/Tools.py:15-55).

Bundled: STO-3G, 6-31G** and 6-31G* (6-31G** without the p polarisation
shells on H and He; the reference has no 6-31G* entry).
"""
import importlib

basis_map = {
    "sto3g": "sto3g",
    "sto-3g": "sto3g",
    "6-31g**": "p631ss",
    "6-31g(d,p)": "p631ss",
    "6-31g*": "p631s",
    "6-31g(d)": "p631s",
}


def get_basis_data(name):
    key = name.lower()
    if key not in basis_map:
        raise KeyError("Can't import basis set %s (bundled: %s)" % (key, ", ".join(sorted(basis_map))))
    return importlib.import_module("pyquante_b200.Basis." + basis_map[key]).basis_data
