// Exact product, factorization and residue-engine kernel instantiations for limb counts 24..25.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(24)
LF_FACTOR_INSTANTIATE(24)
LF_RESIDUE_INSTANTIATE(24)
LF_LINALG_INSTANTIATE(25)
LF_FACTOR_INSTANTIATE(25)
LF_RESIDUE_INSTANTIATE(25)
