// Exact product, factorization and residue-engine kernel instantiations for limb counts 28..29.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(28)
LF_FACTOR_INSTANTIATE(28)
LF_RESIDUE_INSTANTIATE(28)
LF_LINALG_INSTANTIATE(29)
LF_FACTOR_INSTANTIATE(29)
LF_RESIDUE_INSTANTIATE(29)
