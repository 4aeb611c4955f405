/* CPU oracle: PCS parameter ladder and helpers. Test infrastructure only. */
#ifndef BITZ_ORACLE_PCS_H
#define BITZ_ORACLE_PCS_H

#include "oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One Ligerito level (crates/pcs/src/profiles.rs:66-126). */
typedef struct {
  int k;             /* variables folded at this level (log_num_interleaved) */
  int log_inv_rate;  /* code rate 2^-log_inv_rate */
  int log_msg_cols;  /* variables left after the fold */
  int queries;
  int fold_grinding; /* native bits of the first fold; round r uses bits - r */
  int grinding;      /* query grinding bits */
  int ood_samples;   /* recursive out-of-domain samples (Johnson, level > 0) */
} o_pcs_level_t;

typedef struct {
  int m, log_n, security_bits, nlevels, final_log_n;
  o_pcs_level_t levels[8];
} o_pcs_config_t;

int o_pcs_config(int m, int security_bits, o_pcs_config_t *cfg);
o_f128 o_wh(int t, o_f128 x);
void o_rs_encode_column(const o_f128 *msg, size_t stride_in, int l, int d, o_f128 *out,
                        size_t stride_out);
o_f128 o_novel_eval(const o_f128 *c, int l, o_f128 x);
void o_merkle_build(const o_f128 *codeword, size_t rows, int width, uint8_t *nodes);
void o_pcs_encode(const o_f128 *vec, int log_n, int k, int log_inv_rate, o_f128 *codeword);

#ifdef __cplusplus
}
#endif
#endif
