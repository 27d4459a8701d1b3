/*
 * Link stubs for building modpn's CPU FFT multiply (the reference CPU path)
 * without the GPU library.  modpn's FMUL.c asks `can_call_fftmul_uni` before
 * dispatching to the GPU (modpn/src/FMUL.c:1945); answering 0 keeps every
 * product on modpn's own Montgomery FFT (FMUL.c:1757-1809), which is what the
 * oracle and the CPU baseline time.
 *
 * Test infrastructure only: nothing in the shipped library links this file.
 */
#include <stddef.h>

typedef int sfixn;

int can_call_fftmul_uni(sfixn df, sfixn dg) { (void)df; (void)dg; return 0; }

int cumodp_fftmul_uni(sfixn dh, sfixn *H, sfixn df, const sfixn *F,
                      sfixn dg, const sfixn *G, sfixn p)
{
    (void)dh; (void)H; (void)df; (void)F; (void)dg; (void)G; (void)p;
    return 1; /* CUMODP_FAILURE: never taken because can_call_fftmul_uni is 0 */
}
