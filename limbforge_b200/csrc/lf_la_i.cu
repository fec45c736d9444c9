// Exact product, factorization and residue-engine kernel instantiations for limb counts 30..31.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(30)
LF_FACTOR_INSTANTIATE(30)
LF_RESIDUE_INSTANTIATE(30)
LF_LINALG_INSTANTIATE(31)
LF_FACTOR_INSTANTIATE(31)
LF_RESIDUE_INSTANTIATE(31)
