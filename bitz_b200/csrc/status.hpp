// Status codes returned across the C ABI. They mirror the reference's typed
// error enums: tooling/cli/src/end_to_end.rs:58-84 (Error),
// crates/post_gkr/src/lib.rs:47-55 (ProveError), crates/pcs/src/opening.rs
// (ProveError) and crates/prover/src/prove.rs:14-28.
#pragma once

#define BZ_OK 0
#define BZ_ERR_ARGUMENT 1        /* bad sizes or null pointers (Error::Input) */
#define BZ_ERR_CLAIM 2           /* the claimed value does not hold (ClaimDoesNotHold) */
#define BZ_ERR_UNSATISFIED 3     /* witness does not satisfy the constraints */
#define BZ_ERR_CONFIG 4          /* unsupported shape or parameters (Configuration) */
#define BZ_ERR_CUDA 5            /* a CUDA call failed */
#define BZ_ERR_INTERNAL 6        /* an internal consistency check failed */
#define BZ_ERR_SCRATCH 7         /* scratch memory too small for the request */
#define BZ_ERR_VERIFY 8          /* verification rejected the proof */
#define BZ_ERR_MALFORMED 9       /* proof bytes do not decode */
#define BZ_ERR_NO_DEVICE 10      /* no CUDA device is available */
#define BZ_PENDING 11            /* a served request has not finished yet */
