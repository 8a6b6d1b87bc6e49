# Heat/cool test network (HCTOY): a KROME-style Python dump with the KROME
# species layout -- chemical species first, then CR, g, Tgas and a dummy --
# so that the preprocessor's --heatcool=1 replaces the Tgas row by the
# heating/cooling term.  Species: E, H+, H, H2, HE, CR, g, Tgas, dummy.
# Reactions (constant rate coefficients, cm^3/s and 1/s):
#   H + E -> H+ + E + E   1e-15
#   H+ + E -> H           2e-13
#   H + H -> H2           1e-17
#   H2 -> H + H           1e-10
# Defines y, rhs, neq, nrea (the format of the reference's pre_odevec.py:97-105).
neq = 9
nrea = 4
y = [Symbol('y(:,%d)' % (i + 1)) for i in range(neq)]
rhs = Matrix([
    1e-15*y[2]*y[0] - 2e-13*y[1]*y[0],
    1e-15*y[2]*y[0] - 2e-13*y[1]*y[0],
    -1e-15*y[2]*y[0] + 2e-13*y[1]*y[0] - 2*1e-17*y[2]*y[2] + 2*1e-10*y[3],
    1e-17*y[2]*y[2] - 1e-10*y[3],
    0,
    0,
    0,
    0,
    0,
])
