/* Input generators of the reference's GPU bench (host only).
 *
 * brdc_input_generate replaces make_bench_tridiagonal_data,
 * make_paper_tridiagonal_data and make_test_tridiagonal_data
 * (gpu/bench/tridiag_dc_bench.cu:229-339; the bench picks one through its
 * --data option, :1336-1338 and :1504-1521).  It fills D[n] and E[n-1] with
 * the same values, drawn from the same C++ <random> engines with the same
 * seeds.
 *
 * mode   "bench", "test", "normal", "uniform", "toeplitz" or "clustered"
 * index  position of n in the bench's size list ("bench" seeds 1234 + index;
 *        the other modes ignore it)
 *
 * Returns BRDC_INPUT_OK, BRDC_INPUT_UNKNOWN_MODE for any other mode, or
 * BRDC_INPUT_BAD_ARGUMENT for n < 1 or a null pointer (E may be null when
 * n == 1).  Built into libbrdc_inputs.so; needs no GPU.
 */
#ifndef BRDC_INPUTS_H
#define BRDC_INPUTS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    BRDC_INPUT_OK = 0,
    BRDC_INPUT_UNKNOWN_MODE = -1,
    BRDC_INPUT_BAD_ARGUMENT = -2
};

int brdc_input_generate(const char *mode, int64_t n, int64_t index, double *D, double *E);

#ifdef __cplusplus
}
#endif

#endif /* BRDC_INPUTS_H */
