/* or_threads.c -- CPU-baseline driver for the reference Metropolis update.
 *
 * TEST INFRASTRUCTURE ONLY (see or_internal.h): used by bench.py's
 * CPU-baseline leg.  The reference is single threaded (one chain per
 * process, su3_ensemble.rs:408-480), so the multi-core baseline runs one
 * independent chain per thread: each thread owns a cold lattice of the given
 * extents and a SplitMix64 stream derived with derive_su3_chain_seed, and
 * visits `links_per_thread` links in the reference's lexicographic order
 * with the reference's eight ordered generator hits per link
 * (su3_ensemble.rs:355-389).  Wall time is measured around all threads.
 */
#include <pthread.h>
#include <stdlib.h>
#include <time.h>

#include "oracle.h"
#include "or_internal.h"

typedef struct {
    const int64_t *ext;
    double beta, angle;
    uint64_t seed;
    int64_t nlinks;
    double *links;
    uint64_t done;
    int status;
} worker_arg;

static int visit_reference_link(const int64_t *ext, double *links, const int64_t x[4], int mu,
                                double beta, double angle, uint64_t *rng) {
    extents4 e;
    extents_from(ext, &e, 0, NULL);
    int64_t l = site_index(&e, x) * 4 + mu;
    for (int g = 0; g < 8; ++g) {
        double a, coef[8] = {0}, delta;
        int st = or_proposal_angle_from_u64(sm_next(rng), angle, &a);
        if (st) return st;
        coef[g] = a;
        double rot[18], cand[18];
        st = or_su3_from_algebra(coef, rot);
        if (st) return st;
        mat3 r, u, c;
        memcpy(&r, rot, sizeof r);
        u = su3_load(links, l);
        st = su3_mul_checked(r, u, &c);
        if (st) return st;
        memcpy(cand, &c, sizeof c);
        st = or_su3_local_action_difference(ext, links, x, mu, cand, beta, &delta);
        if (st) return st;
        double acc = exp(-fmax(delta, 0.0));
        if (sm_unit(rng) < acc) su3_store(links, l, c);
    }
    return YM_OK;
}

static void *worker(void *p) {
    worker_arg *w = (worker_arg *)p;
    uint64_t rng = w->seed;
    int64_t x[4] = {0, 0, 0, 0};
    int mu = 0;
    for (int64_t k = 0; k < w->nlinks; ++k) {
        w->status = visit_reference_link(w->ext, w->links, x, mu, w->beta, w->angle, &rng);
        if (w->status) return NULL;
        w->done += 1;
        if (++mu == 4) {           /* lexicographic site order, x3 fastest */
            mu = 0;
            for (int d = 3; d >= 0; --d) {
                if (++x[d] < w->ext[d]) break;
                x[d] = 0;
            }
        }
    }
    return NULL;
}

int or_bench_su3_reference(const int64_t *ext, double beta, double angle, uint64_t master_seed,
                           int64_t threads, int64_t links_per_thread, double *seconds,
                           uint64_t *link_updates) {
    extents4 e;
    int64_t nl;
    int st = extents_from(ext, &e, 0, &nl);
    if (st) return st;
    if (threads < 1) return YM_ERR_INVALID_ARGUMENT;
    pthread_t *tid = calloc((size_t)threads, sizeof(pthread_t));
    worker_arg *args = calloc((size_t)threads, sizeof(worker_arg));
    if (!tid || !args) { free(tid); free(args); return YM_ERR_ALLOCATION_FAILED; }
    for (int64_t t = 0; t < threads && !st; ++t) {
        args[t].ext = ext;
        args[t].beta = beta;
        args[t].angle = angle;
        args[t].seed = or_derive_su3_chain_seed(master_seed, (uint64_t)t);
        args[t].nlinks = links_per_thread;
        args[t].links = malloc((size_t)nl * 18 * sizeof(double));
        if (!args[t].links) st = YM_ERR_ALLOCATION_FAILED;
        else or_su3_identity(ext, 1, args[t].links);
    }
    struct timespec t0, t1;
    if (!st) {
        clock_gettime(CLOCK_MONOTONIC, &t0);
        for (int64_t t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, worker, &args[t]);
        for (int64_t t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
        clock_gettime(CLOCK_MONOTONIC, &t1);
        *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
        uint64_t done = 0;
        for (int64_t t = 0; t < threads; ++t) {
            done += args[t].done;
            if (args[t].status) st = args[t].status;
        }
        *link_updates = done;
    }
    for (int64_t t = 0; t < threads; ++t) free(args[t].links);
    free(tid);
    free(args);
    return st;
}
