// Exact product, factorization and residue-engine kernel instantiations for limb counts 32..32.
#include "lf_residue.cuh"
LF_LINALG_INSTANTIATE(32)
LF_FACTOR_INSTANTIATE(32)
LF_RESIDUE_INSTANTIATE(32)
