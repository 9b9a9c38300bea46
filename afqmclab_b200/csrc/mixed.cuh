// Mixed-precision form of the walker step (tensor-core contractions; FP64
// LU/log-determinant, phases, weights and re-orthonormalisation).
#pragma once
struct afqmc_engine;
struct MixedState;

int mixed_create(afqmc_engine *e);
void mixed_destroy(afqmc_engine *e);
int mixed_project_dtk_dtv(afqmc_engine *e);
int mixed_modify_gm(afqmc_engine *e);
int mixed_add_measurement(afqmc_engine *e);
int mixed_update_operators(afqmc_engine *e);
// keep the FP64 walker copy and the reduced-precision working copy in step
int mixed_sync_to_fp64(afqmc_engine *e);
int mixed_sync_from_fp64(afqmc_engine *e);
int mixed_status(afqmc_engine *e);
int mixed_pop_control(afqmc_engine *e);
int mixed_exchange(afqmc_engine *e);
