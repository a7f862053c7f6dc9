/*
 * oracle_common.h -- shared helpers of the CPU oracle.
 *
 * TEST INFRASTRUCTURE. The oracle is the checker of the CUDA library: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs load it.
 * The product path never calls it.
 *
 * The reference (DavRack/imops) is Rust; no Rust toolchain exists where this
 * repository is built, so the oracle restates the reference's arithmetic in C.
 * Files that restate f32 code are compiled with -ffp-contract=off on x86-64
 * (SSE, no excess precision), so each float operation rounds exactly like the
 * reference's f32 operation in the same order.  Files that restate f64 code
 * call glibc's libm, which is what Rust's f64::exp/powf/log10 lower to on
 * Linux.
 *
 * Precision switch: a source including this header is compiled once with
 * ORACLE_F32 (reference order, the parity target) and once without it (an
 * FP64 instantiation of the same steps, used to report error against an
 * FP64 oracle).  OSYM(name) appends _f32 / _f64 to exported symbols and
 * K(x) spells a literal in the working precision.
 */
#ifndef ORACLE_COMMON_H
#define ORACLE_COMMON_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#ifdef ORACLE_F32
typedef float real;
#define K(x) x##f
#define OSYM(n) n##_f32
#define RABS fabsf
#define RMAX fmaxf
#define RMIN fminf
#else
typedef double real;
#define K(x) x
#define OSYM(n) n##_f64
#define RABS fabs
#define RMAX fmax
#define RMIN fmin
#endif

/* Status codes shared with the CUDA library's C-ABI. */
#define ORACLE_OK 0
#define ORACLE_ERR_ARG 1
#define ORACLE_ERR_CFA 2
#define ORACLE_ERR_SIZE 3

/* Colour of a CFA site, the reference's CFA::color_at (cfa.rs:148-150):
 * the pattern repeats with its own period, so a 48x48 table lookup with
 * (r+48)%48 is the same as indexing the period with a positive modulo. */
typedef struct {
    int pw, ph;             /* period width / height */
    uint8_t col[12 * 12];   /* colour per period cell, row-major, 0=R 1=G 2=B */
} OracleCfa;

static inline int ocfa_color(const OracleCfa *c, long r, long q)
{
    long rr = r % c->ph; if (rr < 0) rr += c->ph;
    long cc = q % c->pw; if (cc < 0) cc += c->pw;
    return c->col[rr * c->pw + cc];
}

/* Parallel loop over [0, n) in chunks on `threads` pthreads (the image has
 * no OpenMP runtime).  fn(ctx, worker, begin, end) runs one chunk; `worker`
 * indexes per-thread scratch.  Defined in parallel.c. */
typedef void (*oracle_chunk_fn)(void *ctx, int worker, long begin, long end);
void oracle_parallel_for(long n, long chunk, int threads, oracle_chunk_fn fn, void *ctx);

#endif
