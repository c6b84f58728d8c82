/* The reference-named surface used out of order (sampling before init, NULL arguments) records
 * an error in nmlmc_last_error() and returns instead of exiting or crashing (compiled and run by
 * tests/test_abi.py). */
#include <stdio.h>
#include "nmlmc.h"

int main(void) {
    int bad = 0;
    double f[4] = {0}, d[4] = {0};
    sample_output out = {0, f, d, 0.0, {0}};
    model_sample(2, 10, &out);
    printf("model_sample before init: %d\n", nmlmc_last_error());
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    portfolio_sample(2, 0, 10, &out);
    printf("portfolio_sample before init: %d\n", nmlmc_last_error());
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    init_nestedmc_sampler(4, NULL);
    printf("init with NULL params: %d\n", nmlmc_last_error());
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    model_init(NULL, 0);
    printf("model_init(NULL): %d\n", nmlmc_last_error());
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    model_sample(0, 10, NULL);
    printf("model_sample(NULL out): %d\n", nmlmc_last_error());
    if (nmlmc_last_error() == NMLMC_OK) bad++;
    cleanup_nestedmc_sampler();
    cleanup_nestedmc_sampler();          /* twice: harmless */
    printf("ok-calls %d\n", bad);
    return bad != 0;
}
