/*
 * crush_server.h — continuous-batching crash server on one GPU.
 *
 * No counterpart in the reference, which runs one crash per process
 * (src/bin/crushrs.rs:30). Requests (whole crash models) are submitted from
 * any thread and answered asynchronously. Each serving context is a batched
 * context with room for more crashes (crush_batch_create_reserved), driven
 * in chunks of steps on its own CUDA stream and host thread; between chunks
 * it admits the requests waiting for it into its running batch
 * (crush_batch_append, the new crashes' set-up overlapping the chunk just
 * issued), so a request starts within one chunk of its arrival while the
 * others keep running. A scheduler thread opens a context when requests wait
 * that no open context takes (every context's room spent, or another
 * schedule class) and the HBM budget has room; contexts run side by side on
 * the device. Every crash is reported the moment its own stop rule ends it,
 * and its results are bit-identical to crush_create + crush_run of the same
 * model alone.
 */
#ifndef CRUSH_SERVER_H
#define CRUSH_SERVER_H

#include <stdint.h>

#include "crush.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct crush_server crush_server;

typedef struct crush_server_config {
    int32_t device;
    int32_t max_waves;          /* serving contexts running at once (default 4) */
    int32_t max_wave_slots;     /* crashes a context takes over its life (its slot room, default 1024) */
    int32_t chunk_steps;        /* steps between admissions and completion checks (a multiple of 20, default 100;
                                   20 while requests wait) */
    int64_t max_wave_elements;  /* hexahedra a context takes over its life (its element room, default 2,000,000) */
    double hbm_budget_bytes;    /* device memory the contexts may hold together (0 = 80% of free memory) */
    double gather_ms;           /* while contexts run, a new context waits this long for more arrivals (default 2) */
    double idle_ms;             /* a context with no crash running waits this long for requests before it ends (default 200) */
    int32_t max_queue;          /* admission control: a submit that finds this many requests waiting is refused with
                                   CRUSH_ERR_BUSY, nothing copied (0 = no limit) */
    int32_t max_running;        /* a context with this many crashes running takes no new requests while another
                                   context can be opened (within max_waves); 0 = no limit */
} crush_server_config;

typedef struct crush_server_result {
    uint64_t ticket;
    int32_t status;             /* CRUSH_OK, CRUSH_ERR_NONFINITE, or the error that stopped the wave */
    int32_t wave;               /* index of the serving context that ran it */
    double submit_s;            /* server clock (s since creation) at submit */
    double start_s;             /* admitted into its context's run */
    double finish_s;            /* result available */
    crush_results results;
} crush_server_result;

typedef struct crush_server_stats {
    int64_t submitted, completed, waves, queued, running;  /* waves: serving contexts opened; running: contexts running */
    double bytes_in_use, peak_bytes_in_use, budget_bytes;
} crush_server_stats;

/* config may be NULL (defaults). */
int crush_server_create(const crush_server_config* config, crush_server** out);
/* Copies the model (the caller may free it on return) and queues it;
 * CRUSH_ERR_BUSY when max_queue requests already wait. */
int crush_server_submit(crush_server* srv, const crush_model_desc* desc, uint64_t* ticket);
/* Up to max finished results into out, waiting up to wait_ms for the first. */
int crush_server_poll(crush_server* srv, crush_server_result* out, int max, int* n, int wait_ms);
int crush_server_stats_get(crush_server* srv, crush_server_stats* out);
/* Estimated device bytes of a model inside a wave (the admission measure). */
double crush_model_footprint(const crush_model_desc* desc);
/* Finishes every submitted request, then stops the server's threads. */
void crush_server_destroy(crush_server* srv);

#ifdef __cplusplus
}
#endif
#endif
