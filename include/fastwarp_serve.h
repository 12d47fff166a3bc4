/*
 * fastwarp_serve.h -- continuous-batching registration server on one GPU.
 *
 * The reference runs several registrations on one device at once only in `register_atlases`
 * (crates/fastwarp-cli/src/engine.rs:1016-1072: up to four at a time, admitted by a memory
 * budget). This server generalises that path: requests of any grid size arrive at any time, are
 * admitted as soon as an execution slot is free and their device-memory estimate fits the HBM
 * budget, and then run concurrently -- each on its own context and stream, each level of each
 * registration one CUDA graph -- so their kernels overlap on the GPU. Results do not depend on
 * what else is running: every kernel is deterministic and no state is shared between requests.
 */
#ifndef FASTWARP_SERVE_H
#define FASTWARP_SERVE_H

#include "fastwarp_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fw_server fw_server;

/* One SyN-stage request (run_syn, syn.rs:555-564). Images are either host float32 volumes
 * (copied at submit, so the caller may free them at once) or device images made on any context
 * of the same device (used in place; they must stay alive until the request completes, and
 * their contents must be complete when submitted: the slot reads them on its own stream without
 * waiting for the caller's, so a caller that filled them asynchronously synchronises first). */
typedef struct fw_syn_request {
    fw_syn_recipe recipe;
    fw_grid fixed_grid;
    fw_grid moving_grid;
    const float* const* fixed;         /* host, one per channel, or NULL */
    const float* const* moving;
    const fw_image* const* fixed_dev;  /* device, one per channel, or NULL */
    const fw_image* const* moving_dev;
    fw_affine initial;
    int32_t has_initial;
    int32_t keep_on_device;  /* 1: the fields stay on the device (warp_dev / inverse_dev) */
    uint64_t tag;
    /* The recipe's masks (recipe.rs fixed_mask / moving_mask), each on its own grid: host float32
     * data (copied at submit) or a device image (kept valid until the result is taken); both
     * NULL when the mask is not given. */
    fw_grid fixed_mask_grid;
    fw_grid moving_mask_grid;
    const float* fixed_mask;
    const float* moving_mask;
    const fw_image* fixed_mask_dev;
    const fw_image* moving_mask_dev;
} fw_syn_request;

typedef struct fw_syn_result {
    uint64_t tag;
    int32_t status;            /* FW_OK or an FW_ERR_* code */
    char error[256];
    fw_grid grid;              /* the last level grid of the fields */
    float* warp;               /* host AoS float32 (keep_on_device == 0), else NULL */
    float* inverse_warp;
    fw_field* warp_dev;        /* keep_on_device == 1; free with fw_field_free before the server */
    fw_field* inverse_dev;
    int64_t iterations;
    double final_energy;
    uint64_t device_bytes;     /* the admission estimate of this request */
    double queued_s;           /* submit -> start (host clock) */
    double run_s;              /* start -> done (host clock) */
    double device_start_ms;    /* device clock, relative to the last fw_server_mark */
    double device_end_ms;
} fw_syn_result;

/* One linear-stage request (run_linear_stage, linear.rs:512-597; the reference's affine-only
 * registrations): host float32 images (copied at submit) or device images made on any context of
 * the same device (kept alive until the result is taken, and complete when submitted, as for a
 * SyN request). `start` is the start transform, with the earlier transforms as its outer part. */
typedef struct fw_linear_request {
    fw_linear_recipe recipe;
    fw_grid fixed_grid;
    fw_grid moving_grid;
    const float* fixed;                /* host, or NULL */
    const float* moving;
    const fw_image* fixed_dev;         /* device, or NULL */
    const fw_image* moving_dev;
    fw_linear_transform start;
    uint64_t tag;
} fw_linear_request;

typedef struct fw_linear_result {
    uint64_t tag;
    int32_t status;                    /* FW_OK or an FW_ERR_* code */
    char error[256];
    fw_linear_transform transform;     /* the optimised transform */
    int32_t nlevels;
    fw_linear_level_trace levels[FW_MAX_LEVELS];
    uint64_t device_bytes;             /* the admission estimate of this request */
    double queued_s;                   /* submit -> start (host clock) */
    double run_s;                      /* start -> done (host clock) */
} fw_linear_result;

typedef struct fw_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t active, queued;
    uint64_t reserved_bytes, peak_reserved_bytes, budget_bytes;
    uint64_t kernel_launches, graph_launches;
} fw_server_stats;

/* A server on `device` with `slots` execution slots (each its own context and stream) that
 * admits requests while the sum of their device-memory estimates stays within `hbm_budget`
 * bytes (0: 90 % of the device's free memory). */
int fw_server_create(int device, uint64_t hbm_budget, int32_t slots, fw_server** out);
/* Queues a request; returns at once with its ticket. Fails with FW_ERR_MEMORY when the request
 * alone exceeds the budget. */
int fw_server_submit(fw_server* s, const fw_syn_request* req, uint64_t* ticket);
/* Waits for a ticket (timeout_s < 0: forever) and moves its result to `out`; FW_ERR_TIMEOUT when
 * it is not done in time. A ticket's result can be taken once. */
int fw_server_wait(fw_server* s, uint64_t ticket, double timeout_s, fw_syn_result* out);
/* Frees the host buffers of a result (not the device fields). */
void fw_server_result_free(fw_syn_result* r);
/* Records the device-clock origin of device_start_ms / device_end_ms. */
int fw_server_mark(fw_server* s);
int fw_server_stats_get(fw_server* s, fw_server_stats* out);
/* The device-memory estimate the server admits a request by. */
int fw_server_estimate(const fw_syn_request* req, uint64_t* bytes);
/* Linear-stage requests share the slots, the queue and the HBM budget with SyN requests; a
 * ticket is waited for with the function of its kind (the other one fails). */
int fw_server_submit_linear(fw_server* s, const fw_linear_request* req, uint64_t* ticket);
int fw_server_wait_linear(fw_server* s, uint64_t ticket, double timeout_s, fw_linear_result* out);
int fw_server_estimate_linear(const fw_linear_request* req, uint64_t* bytes);
/* Cancels a request of either kind (SynOptions::cancel, syn.rs:80-85): a queued one ends at once
 * without running; a running one stops after the SyN iteration (or linear-optimiser iteration)
 * in flight, through its slot context's cancel flag, which the level graph reads once per
 * iteration. Either way its result carries FW_ERR_CANCELLED; the other requests run on untouched.
 * A request that has finished keeps its result. The ticket is still waited for as usual. */
int fw_server_cancel(fw_server* s, uint64_t ticket);
/* Waits for every queued and running request, then stops the slots. */
void fw_server_destroy(fw_server* s);

/* No counterpart in the reference: sizeof of a struct of these headers by name ("fw_grid",
 * "fw_syn_recipe", "fw_syn_request", ...; 0 for an unknown name), for bindings to check their
 * mirrored layouts against the library's. */
size_t fw_abi_struct_size(const char* name);

#ifdef __cplusplus
}
#endif
#endif
