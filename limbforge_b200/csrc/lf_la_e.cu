// Exact product, factorization and residue-engine kernel instantiations for limb counts 22..23.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(22)
LF_FACTOR_INSTANTIATE(22)
LF_RESIDUE_INSTANTIATE(22)
LF_LINALG_INSTANTIATE(23)
LF_FACTOR_INSTANTIATE(23)
LF_RESIDUE_INSTANTIATE(23)
