/*
 * One cumodp_fftmul_uni_dev call per product, in a compiled C loop: the
 * plain one-call-per-product path that the batched entry point is measured
 * against, without an interpreter between the calls.  Built next to
 * libcumodp.so by cumodp_b200/build.py (libcumodp_percall.so) and loaded by
 * bench.py.
 */
#include <stdint.h>

#include "cumodp.h"

/* Products i < count: H + h_off[i] (df[i] + dg[i] + 1 words) =
 * (F + f_off[i]) * (G + g_off[i]) mod p, device pointers, all on `stream`
 * (asynchronous: the caller synchronises).  Returns the first error. */
int percall_fftmul(int count, const sfixn *df, const int64_t *f_off, const sfixn *F, const sfixn *dg,
                   const int64_t *g_off, const sfixn *G, const int64_t *h_off, sfixn *H, sfixn p, void *stream)
{
    for (int i = 0; i < count; ++i) {
        cumodp_err e = cumodp_fftmul_uni_dev(df[i] + dg[i] + 1, H + h_off[i], df[i], F + f_off[i], dg[i],
                                             G + g_off[i], p, stream);
        if (e != CUMODP_SUCCESS) return (int)e;
    }
    return 0;
}
