"""Element symbols and numbers for Z = 1..18 (the elements the bundled basis
sets cover); mirrors the name2no/sym2no maps of PyQuante/Element.py."""
symbol = [None, "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne",
          "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]
sym2no = {s: z for z, s in enumerate(symbol) if s}
sym2no.update({s.upper(): z for z, s in enumerate(symbol) if s})
name2no = dict(sym2no)
