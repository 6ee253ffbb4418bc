"""Physical constants in eV, Angstrom, K and e (src/constants.jl:3-4)."""

# Boltzmann constant in eV/K and the Coulomb prefactor 1/(4 pi eps0) in eV*A/e^2, CODATA 2014 as
# used by kUPS.
KB = 1.38064852e-23 / 1.6021766208e-19
KE = 14.399645351950548
