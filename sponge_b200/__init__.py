"""B200-native (sm_100a) nonbonded hot path of SPONGE: neighbor list,
LJ + erfc-Coulomb pair kernel (and soft-core variant), smooth-PME reciprocal
part and the force / energy / virial reductions, behind the C ABI in
include/sponge_nb.h.  ``capi`` is the ctypes binding; ``systems`` builds the
seeded water / NaCl boxes the benchmarks and tests use."""

__all__ = ["capi", "systems", "build"]
