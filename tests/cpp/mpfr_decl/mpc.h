/* TEST INFRASTRUCTURE ONLY: the mpc_t layout from the public GNU MPC manual (a pair of mpfr_t), for the bridge test in
 * an image without MPC headers.  The bridge uses no libmpc function. */
#ifndef LIMBFORGE_TEST_MPC_DECL_H
#define LIMBFORGE_TEST_MPC_DECL_H
#include "mpfr.h"
typedef struct { mpfr_t re; mpfr_t im; } __mpc_struct;
typedef __mpc_struct mpc_t[1];
typedef __mpc_struct* mpc_ptr;
typedef const __mpc_struct* mpc_srcptr;
#define mpc_realref(x) ((x)->re)
#define mpc_imagref(x) ((x)->im)
#endif
