/*
 * A thin C driver over modpn's CPU FFT multiply, compiled together with the
 * reference's own modpn sources (see Makefile).  This is the reference CPU
 * implementation of the product path: `EX_Mont_FFTMul`
 * (modpn/src/FMUL.c:2015-2030) dispatches to the plain product below degree
 * 138 (FMUL.h:36) and otherwise to the Montgomery radix-2 DFT / pairwise /
 * inverse DFT of FMUL.c:1757-1809.
 *
 * Test infrastructure only: used by tests/ as an independent checker and by
 * bench.py as the timed reference arm / CPU baseline.
 */
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include "Types.h"
#include "FMUL.h"

void EX_MontP_Init_OPT2_AS_GENE(MONTP_OPT2_AS_GENE *pPtr, sfixn p);

/* Prime structures are initialised once per prime, before any threading:
 * EX_MontP_Init_OPT2_AS_GENE draws a root with rand() (FMUL.c:59-71). */
#define REF_MAX_PRIMES 16
static MONTP_OPT2_AS_GENE g_primes[REF_MAX_PRIMES];
static sfixn g_prime_vals[REF_MAX_PRIMES];
static int g_nprimes = 0;

static MONTP_OPT2_AS_GENE *prime_struct(sfixn p)
{
    for (int i = 0; i < g_nprimes; ++i)
        if (g_prime_vals[i] == p) return &g_primes[i];
    return NULL;
}

/* Returns 0 on success, -1 if the table is full. Not thread-safe: call it
 * from one thread for every prime before calling ref_fftmul concurrently. */
int ref_init_prime(sfixn p)
{
    if (prime_struct(p)) return 0;
    if (g_nprimes >= REF_MAX_PRIMES) return -1;
    EX_MontP_Init_OPT2_AS_GENE(&g_primes[g_nprimes], p);
    g_prime_vals[g_nprimes] = p;
    ++g_nprimes;
    return 0;
}

/* H (da+db+1 words) = A (da+1) * B (db+1) mod p.  Returns 0 on success,
 * -1 if the prime was not initialised, -2 if modpn flagged a prime error
 * (transform size above the prime's 2-adic order). */
int ref_fftmul(sfixn da, const sfixn *A, sfixn db, const sfixn *B, sfixn *H, sfixn p)
{
    MONTP_OPT2_AS_GENE *pp = prime_struct(p);
    if (!pp) return -1;
    sfixn dr = da + db;
    memset(H, 0, sizeof(sfixn) * (size_t)(dr + 1));
    /* modpn takes non-const pointers but only reads A and B. */
    EX_Mont_FFTMul(dr, H, da, (sfixn *)A, db, (sfixn *)B, pp);
    return 0;
}

/* `count` independent products spread over `threads` POSIX threads, one
 * product per thread at a time (work is handed out through an atomic
 * counter).  Operand i lives at A + a_off[i] (da[i]+1 words), B + b_off[i]
 * (db[i]+1 words); its result goes to H + h_off[i] (da[i]+db[i]+1 words).
 * Returns the number of failed products. */
typedef struct {
    int count; const sfixn *da; const long *a_off; const sfixn *A;
    const sfixn *db; const long *b_off; const sfixn *B;
    const long *h_off; sfixn *H; sfixn p;
    int next; int fails;
} batch_job;

static void *batch_worker(void *arg)
{
    batch_job *j = (batch_job *)arg;
    for (;;) {
        int i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (i >= j->count) break;
        if (ref_fftmul(j->da[i], j->A + j->a_off[i], j->db[i], j->B + j->b_off[i],
                       j->H + j->h_off[i], j->p) != 0)
            __atomic_fetch_add(&j->fails, 1, __ATOMIC_RELAXED);
    }
    return NULL;
}

int ref_fftmul_batch(int count, const sfixn *da, const long *a_off, const sfixn *A,
                     const sfixn *db, const long *b_off, const sfixn *B,
                     const long *h_off, sfixn *H, sfixn p, int threads)
{
    if (!prime_struct(p)) return count;
    batch_job job = {count, da, a_off, A, db, b_off, B, h_off, H, p, 0, 0};
    if (threads < 1) threads = 1;
    if (threads > 1024) threads = 1024;
    pthread_t tid[1024];
    int started = 0;
    for (int t = 1; t < threads; ++t)
        if (pthread_create(&tid[started], NULL, batch_worker, &job) == 0) ++started;
    batch_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    return job.fails;
}
