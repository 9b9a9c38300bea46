// Mixed-precision form (work in progress): not yet constructible.
#include <string>

#include "../../include/afqmc_b200.h"
#include "mixed.cuh"

int mixed_create(afqmc_engine *) { return AFQMC_ERR_UNSUPPORTED; }
void mixed_destroy(afqmc_engine *) {}
int mixed_project_dtk_dtv(afqmc_engine *) { return AFQMC_ERR_UNSUPPORTED; }
int mixed_modify_gm(afqmc_engine *) { return AFQMC_ERR_UNSUPPORTED; }
int mixed_add_measurement(afqmc_engine *) { return AFQMC_ERR_UNSUPPORTED; }
int mixed_update_operators(afqmc_engine *) { return AFQMC_ERR_UNSUPPORTED; }
int mixed_sync_to_fp64(afqmc_engine *) { return AFQMC_OK; }
int mixed_sync_from_fp64(afqmc_engine *) { return AFQMC_OK; }
int mixed_status(afqmc_engine *) { return 0; }
