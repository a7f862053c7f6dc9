/*
 * parallel.c -- pthread parallel-for used by the CPU oracle (test
 * infrastructure, see oracle_common.h).  Chunks are handed out through an
 * atomic counter so uneven work (edge tiles) balances across threads.
 */
#include "oracle_common.h"

#include <pthread.h>

typedef struct {
    long n, chunk;
    long next;
    oracle_chunk_fn fn;
    void *ctx;
} Pool;

typedef struct {
    Pool *pool;
    int worker;
} Arg;

static void *run(void *p)
{
    Arg *a = (Arg *)p;
    Pool *pool = a->pool;
    for (;;) {
        long b = __atomic_fetch_add(&pool->next, pool->chunk, __ATOMIC_RELAXED);
        if (b >= pool->n) break;
        long e = b + pool->chunk < pool->n ? b + pool->chunk : pool->n;
        pool->fn(pool->ctx, a->worker, b, e);
    }
    return NULL;
}

void oracle_parallel_for(long n, long chunk, int threads, oracle_chunk_fn fn, void *ctx)
{
    if (n <= 0) return;
    if (chunk < 1) chunk = 1;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    Pool pool = {n, chunk, 0, fn, ctx};
    pthread_t tid[256];
    Arg args[256];
    for (int i = 0; i < threads; i++) {
        args[i].pool = &pool;
        args[i].worker = i;
    }
    if (threads == 1) {
        run(&args[0]);
        return;
    }
    int started = 0;
    for (int i = 1; i < threads; i++) {
        if (pthread_create(&tid[i], NULL, run, &args[i]) != 0) break;
        started = i;
    }
    run(&args[0]);
    for (int i = 1; i <= started; i++) pthread_join(tid[i], NULL);
}
