/* Every native entry point called with a NULL context or NULL required pointers returns an
 * error status instead of crashing (compiled and run by tests/test_abi.py; no device needed). */
#include <stdio.h>
#include "nmlmc.h"
#define CHECK(call) do { int rc_ = (call); printf("%-40s %d\n", #call, rc_); if (rc_ == NMLMC_OK) bad++; } while (0)
int main(void) {
    int bad = 0;
    nmlmc_config cfg = {0};
    nmlmc_level_result r;
    nmlmc_phase_config pc;
    nmlmc_mlmc_input in = nmlmc_mlmc_default_input();
    nmlmc_mlmc_output out;
    uint32_t ells[1] = {0};
    uint64_t Ms[1] = {10}, u = 0;
    double d = 0;
    size_t sz = 0;
    char buf[16];
    CHECK(nmlmc_configure(NULL, &cfg));
    CHECK(nmlmc_set_model(NULL, NMLMC_MODEL_SHIFT, 0.0, 1.0));
    CHECK(nmlmc_set_portfolio(NULL, NULL, NULL, NULL));
    CHECK(nmlmc_set_portfolio_methods(NULL, NULL, NULL, NULL, NULL));
    CHECK(nmlmc_path_adjoint(NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL));
    CHECK(nmlmc_reset_streams(NULL));
    CHECK(nmlmc_sample(NULL, 0, 10, &r));
    CHECK(nmlmc_sample_levels(NULL, 1, ells, Ms, &r));
    CHECK(nmlmc_set_autotune(NULL, 1));
    CHECK(nmlmc_get_phase_config(NULL, 0, &pc));
    CHECK(nmlmc_set_phase_config(NULL, 0, &pc));
    CHECK(nmlmc_autotune_level(NULL, 0, 100));
    CHECK(nmlmc_graph_stats(NULL, &u, &u, &u));
    CHECK(nmlmc_set_trace(NULL, NULL, 0));
    CHECK(nmlmc_portfolio_full_loss(NULL, 0, 0, 1, &d));
    CHECK(nmlmc_set_shard(NULL, 0, 1));
    CHECK(nmlmc_set_profiling(NULL, 1));
    CHECK(nmlmc_phase_kernel_time(NULL, &u, &d));
    CHECK(nmlmc_mlmc_run(NULL, &in, &out, buf, sizeof buf));
    CHECK(nmlmc_mlmc_run_ckpt(NULL, &in, "x.ckpt", 0, &out, buf, sizeof buf));
    CHECK(nmlmc_get_sampler_state(NULL, NULL, 0, &sz));
    CHECK(nmlmc_set_sampler_state(NULL, buf, sizeof buf));
    CHECK(nmlmc_mlmc_run_cb(NULL, NULL, NULL, NULL, &out, buf, sizeof buf));
    CHECK(nmlmc_mlmc_run_cb(&in, NULL, NULL, NULL, &out, buf, sizeof buf));
    CHECK(nmlmc_mlmc_run_cb_ckpt(&in, NULL, NULL, NULL, NULL, &out, buf, sizeof buf));
    CHECK(nmlmc_create(NULL, 0));
    CHECK(nmlmc_threefry_blocks(NULL, NULL, NULL, 1));
    CHECK(nmlmc_outer_normals(NMLMC_PREC_FP32, 0, 0, 0, 1, NULL));
    CHECK(nmlmc_norm_cdf_fast(NULL, NULL, 1));
    CHECK(nmlmc_portfolio_generate(NULL, 0, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL));
    CHECK(nmlmc_sample_level_noalloc(NMLMC_MODEL_SHIFT, 0, 1, 32, 2, 1.5, 0, NMLMC_PREC_FP32, 0, 0, 0, 10, NULL, NULL));
    printf("ok-calls %d\n", bad);
    return bad != 0;
}
