// Internal interface of the batched engine (jt_batch.cu) used by the
// single-box handle (jt_api.cu): an accurate-mode handle is a batch of one box
// whose particle buffers it fills and reads itself.
#pragma once
#include "jt_internal.cuh"

// Persistent device state of one box of a batch.  The reorder of every force
// pass moves the state into the b-buffers and the host swaps the pointers, so
// callers must re-read pos/vel/id after each pass.
struct jt_box_state {
    jt_config cfg;
    int64_t n[2] = {0, 0};
    float mass[2] = {0.f, 0.f};
    float4 *pos[2] = {}, *vel[2] = {}, *acc[2] = {}, *pos_b[2] = {}, *vel_b[2] = {};
    int *id[2] = {}, *id_b[2] = {};
    float4* tabs = nullptr;      // per-axis k tables (2M float4)
    bool acc_valid = false;      // acc belongs to the current positions
    // Yukawa screening of opposite-species pairs (jt_batch_set_screening):
    // kappa = 1 / lambda (0: none) and the short-range split-factor table
    // of b = kappa r_s (the log table, JT_LTAB_N float2)
    double kappa = 0.0;
    float2* ytab = nullptr;
    int M = 0, order = 3, ngrid = 2;
    size_t bytes = 0;            // device bytes held by this box
    // near-field cells per axis that the box's first force-only pass timed
    // fastest (0: not timed; the default L / r_cut is used)
    int cell_nb = 0;
};

// Per-box step arguments of a batched force pass (kick fused into the walk).
struct jt_box_step {
    float dt;       // the box's step; kicks/drifts apply a fraction of it
    float drag;     // H * dtau_per_dt
};

// Allocate a box whose particle arrays the caller fills (pos/vel/id on the
// batch's stream); n_p + n_m > 0.  The config must be ACCURATE.
int jtb_add_empty(jt_batch* B, const jt_config* cfg, int64_t n_p, int64_t n_m, int* box_id);
jt_box_state* jtb_box(jt_batch* B, int box_id);
// the batch's asynchronous-checkpoint state (jt_ckpt.cu), released on destroy
struct jt_ckpt;
jt_ckpt** jtb_ckpt_slot(jt_batch* B);
// Whether the batch's first force-only pass of a large box may time the
// near-field cell count (tune_cells in jt_batch.cu; on by default).  The
// server turns it off: a request must not wait for the timing runs.
void jtb_set_cell_tune(jt_batch* B, bool on);
void jt_ckpt_release(jt_ckpt* c);
cudaStream_t jtb_stream(jt_batch* B);
// Enqueue one force pass (sort, trees, PM, walk) over the listed boxes;
// kick_frac != 0 fuses the closing kick (kick_frac * dt) into the walk.  No
// host synchronisation; stage times are added to the batch's timings when
// jtb_finish is called.
int jtb_force_pass(jt_batch* B, const int* ids, int n_ids, int parts, float kick_frac,
                   const jt_box_step* steps);
// Synchronise, read the device error word and add the pass's stage times.
int jtb_finish(jt_batch* B);
void jtb_reset_timings(jt_batch* B);
int64_t jtb_phase(jt_batch* B, int i);
// Set a box's accelerations (species AoS float3 in the caller's order, host
// or device) and mark them valid for its current positions; used to restore
// a box that was moved to host memory without recomputing its forces.
// A handle's config, per-species particle masses and the signs of its
// caller-order array (jt_api.cu)
int jth_scale_velocities(jt_handle* h, float a);
int jth_info(jt_handle* h, jt_config* cfg, float* m_plus, float* m_minus, int8_t* signs);
// FP64 diagnostics of one state (jt_diag.cu)
int jt_diag_state(const float4* const pos[2], const float4* const vel[2], const int64_t n[2],
                  const float mass[2], double L, int n_cells, cudaStream_t st, jt_diag* out);
int jtb_set_accel(jt_batch* B, int box_id, const float* acc_p, const float* acc_m, int mem);
// The serving loop's transfers between a box and pinned host arrays (AoS
// float3 per species, the caller's order), queued on the batch's stream with
// no host synchronisation.  The pointers are the DEVICE addresses of pinned
// host memory (cudaHostGetDevicePointer): the gather/scatter kernels read and
// write the host arrays over the bus directly, so no staging buffer is held
// per transfer and several admissions and evictions can be in flight behind
// a step.  The host may read or reuse the arrays only after synchronising
// the stream.  upload: pos required, vel (NULL: zero) and acc (NULL: none;
// else the box's forces become valid) optional.  download: acc is written
// only when the box holds valid forces (*acc_copied says).  remove_async:
// frees the box's memory in stream order (no host wait).
int jtb_upload_async(jt_batch* B, int box_id, const float* const pos[2], const float* const vel[2],
                     const float* const acc[2]);
int jtb_download_async(jt_batch* B, int box_id, float* const pos[2], float* const vel[2], float* const acc[2],
                       bool* acc_copied);
int jtb_remove_async(jt_batch* B, int box_id);
// Map `bytes` of device memory into the batch's pool (one allocation, freed
// at once: the pool keeps it) so that later allocations need no new mapping.
int jtb_reserve(jt_batch* B, size_t bytes);
// One KDK step of one box whose state the host holds between steps: the
// caller-order host arrays (pos, vel, acc per species; pinned for full
// speed) are uploaded into the box (which takes the caller's order), the box
// takes one step, and the arrays are overwritten with the new state.  The
// positions are final after the drift: they are copied back on a side
// stream while the force pass runs.
int jtb_step_host(jt_batch* B, int box_id, float* const pos[2], float* const vel[2], float* const acc[2],
                  float dt, float drag);
