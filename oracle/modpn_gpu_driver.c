/*
 * Drop-in check: modpn's own FFT multiply compiled WITH its GPU dispatch
 * (-D_cuda_modp_, modpn/src/FMUL.c:1943-1957) and linked against this
 * repository's libcumodp.so instead of the reference library.  For products
 * with transform size >= 2^16, EX_KN_Mont_FFTMul_OPT2_AS_GENE_1 calls
 * can_call_fftmul_uni and then cumodp_fftmul_uni(n1 - 1, A, degA, A, degB,
 * B, p) in place, exactly as modpn does.
 *
 * Test infrastructure only (built by `make -C oracle modpn_gpu`).
 */
#include <stdlib.h>
#include <string.h>
#include "Types.h"
#include "FMUL.h"

void EX_MontP_Init_OPT2_AS_GENE(MONTP_OPT2_AS_GENE *pPtr, sfixn p);
/* modpn error flags (modpn/src/generalFuncs.c:25-26) */
extern sfixn Interrupted, PrimeError;

static int ceil_log2(long v) { int e = 0; while ((1L << e) < v) ++e; return e; }

/* H (da+db+1 words) = A * B mod p through modpn's in-place GPU-dispatching
 * product.  Returns 0 on success, -1 on a prime error. */
int modpn_gpu_fftmul(sfixn da, const sfixn *A, sfixn db, const sfixn *B, sfixn *H, sfixn p)
{
    MONTP_OPT2_AS_GENE pr;
    EX_MontP_Init_OPT2_AS_GENE(&pr, p);
    sfixn dr = da + db;
    sfixn e = ceil_log2((long)dr + 1);
    sfixn n = (sfixn)1 << e;
    sfixn *a = (sfixn *)calloc(n, sizeof(sfixn));
    sfixn *b = (sfixn *)calloc(n, sizeof(sfixn));
    sfixn *roots = (sfixn *)calloc(n, sizeof(sfixn));
    memcpy(a, A, sizeof(sfixn) * (size_t)(da + 1));
    memcpy(b, B, sizeof(sfixn) * (size_t)(db + 1));
    EX_Mont_GetNthRoots_OPT2_AS_GENE(e, n, roots, &pr);
    Interrupted = 0;
    PrimeError = 0;
    EX_KN_Mont_FFTMul_OPT2_AS_GENE_1(n, e, dr, roots, da, a, db, b, &pr);
    int rc = PrimeError ? -1 : 0;
    memcpy(H, a, sizeof(sfixn) * (size_t)(dr + 1));
    free(a);
    free(b);
    free(roots);
    return rc;
}
