// Mixed-precision form of the constrained-path (Hubbard) walker step:
// tcgen05 kind::tf32 contractions with compensated (hi + lo) operands,
// FP64 LU/log-determinant, weights, re-orthonormalisation and measurement.
#pragma once
#include <string>

struct afqmc_engine;
struct CpMixedState;

bool cp_mixed_supported(int L, int N, std::string *why);
int cp_mixed_create(afqmc_engine *e);
void cp_mixed_destroy(afqmc_engine *e);
int cp_mixed_project_dtk_dtv(afqmc_engine *e);
int cp_mixed_modify_gm(afqmc_engine *e);
int cp_mixed_pop_control(afqmc_engine *e);
int cp_mixed_pop_weights(afqmc_engine *e);
int cp_mixed_sync_to_fp64(afqmc_engine *e);
int cp_mixed_sync_from_fp64(afqmc_engine *e);
int cp_mixed_status(afqmc_engine *e);
