// Exact product, factorization and residue-engine kernel instantiations for limb counts 26..27.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(26)
LF_FACTOR_INSTANTIATE(26)
LF_RESIDUE_INSTANTIATE(26)
LF_LINALG_INSTANTIATE(27)
LF_FACTOR_INSTANTIATE(27)
LF_RESIDUE_INSTANTIATE(27)
