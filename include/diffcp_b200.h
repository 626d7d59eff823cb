/*
 * diffcp_b200 -- C ABI of the B200 (sm_100a) differentiable codimensional-cloth
 * MPM substep, its adjoint and the Chamfer loss, batched over cloth instances.
 *
 * The reference (denzelzheng/diffcp) has no FFI: its boundary is the Python
 * module surface of src/simulation.py and src/parameter_fitting_functions.py,
 * driven by Taichi kernels.  Each entry point below names the reference
 * function(s) whose work it performs.  diffcp_b200/native.py binds these with
 * ctypes and diffcp_b200/reference_api.py re-exports the reference names.
 *
 * Conventions
 *   - All array arguments are DEVICE pointers owned by the caller, except where
 *     a parameter says "host".  The library never allocates device memory: the
 *     caller provides the static-table and scratch buffers sized by dcp_plan.
 *   - Work is enqueued on `stream` (a cudaStream_t passed as void*; NULL is the
 *     legacy default stream).  Calls on one batch are not thread-safe.
 *   - Every function returns DCP_OK (0) or an error code; dcp_last_error()
 *     returns the message of the last failure on the calling thread.
 *   - Arrays are structure-of-arrays, component-major: a [k][N] array stores
 *     component c of item i at c*N + i.  Particle and target arrays concatenate
 *     all instances in instance order.
 *
 * State snapshot (floats, dcp_plan().state_floats), relative to the rest
 * configuration so that float32 resolves small strains:
 *   [15][Nv] vertices  u(3) v(3) C(9, row-major)   u = x - x0
 *   [18][Nt] triangles C(9) delta3(3) xc(3) vc(3)
 *                      delta3 = d3 - n0, d3 the advected third column of d
 *                      (columns 1-2 of d are the current edges); xc, vc the
 *                      centroid's absolute position and velocity (the
 *                      reference's quadrature_x / quadrature_v, simulation.py:
 *                      390-393), written with every state from its vertices
 *                      (a caller that edits a state's vertex displacements or
 *                      velocities directly must update these to match)
 *   [15][No] operator particles u v C
 *   [15][Nc] cube particles     u v C
 * Rest buffer (floats, dcp_plan().rest_floats), written by dcp_init_state:
 *   [9][Nt] D0^-1, [3][Nt] n0, [6][Nt] rest edges (D0's first two columns),
 *   [3][Nt] rest centroids, [3][Nv] x0, [3][No] x0, [3][Nc] x0
 * Parameter table: [n_inst][8] floats: E, nu, shearing_stiffness,
 *   contact_stiffness, ground friction, damping, 0, 0.
 * Parameter gradients: [n_inst][8] doubles in the same order (accumulated).
 * Trajectory table (floats, per instance, concatenated):
 *   gripper_mode 1: keyframes [n_actions][n_grippers][3]
 *   gripper_mode 2: velocities [n_traj_steps][n_grippers][3] followed by
 *                   centres    [n_traj_steps][n_grippers][3]
 * Trajectory gradients: doubles, same layout (accumulated; centres get none).
 */
#ifndef DIFFCP_B200_H
#define DIFFCP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DCP_OK 0
#define DCP_ERR_INVALID 1
#define DCP_ERR_CUDA 2

#define DCP_GRIP_NONE 0
#define DCP_GRIP_OPERATOR 1  /* heavy operator particles driven by keyframes (simulation.py:154-174) */
#define DCP_GRIP_KINEMATIC 2 /* grid nodes inside a sphere take the gripper velocity (no reference counterpart) */

#define DCP_SVD_GRAD_EXACT 0     /* closed-form derivative of the in-plane rotation factor */
#define DCP_SVD_GRAD_REFERENCE 1 /* clamped SVD backward of simulation.py:44-50,71-94 */

#define DCP_STATUS_OUT_OF_DOMAIN 1 /* a stencil left the grid; clamped */
#define DCP_STATUS_NONFINITE 2     /* a particle velocity became NaN/Inf, or a Chamfer distance was NaN */
#define DCP_STATUS_POOL_FULL 4     /* paged grids: a substep touched more blocks than the pool holds; the
                                      results of that substep are wrong */

/* One cloth scene; the scalars are the constants of src/initialization.py:79,115-130. */
typedef struct DcpInstance {
  int32_t n_vertex, n_tri, n_operator, n_cube, n_target;
  int32_t n_grid;          /* nodes per axis, dx = 1/n_grid (initialization.py:79) */
  int32_t bound;           /* wall layers (initialization.py:22) */
  float vertex_p_mass;     /* initialization.py:130 */
  float quadrature_p_mass; /* initialization.py:129 */
  float quadrature_p_vol;  /* initialization.py:127 */
  float operator_p_mass;   /* initialization.py:125 */
  float cube_p_mass;       /* initialization.py:123 */
  float gravity_dv;        /* dt*scene_scaling*gravity added to vertex velocities (simulation.py:182) */
  int32_t gripper_mode;    /* DCP_GRIP_* */
  int32_t n_grippers;      /* grasp points (mode 1) or spheres (mode 2) */
  int32_t group_size;      /* operator particles per grasp point (initialization.py:164) */
  int32_t n_actions;       /* keyframes (initialization.py:102) */
  float keyframe_interval; /* operator_update_interval (initialization.py:30) */
  int32_t frames_per_window; /* int(grad_update_interval / operator_update_interval) (simulation.py:161) */
  float gripper_radius;    /* mode 2 */
  int32_t n_traj_steps;    /* mode 2 */
} DcpInstance;

typedef struct DcpOptions {
  float dt;            /* substep (initialization.py:31) */
  int32_t chunk;       /* particles per CTA: multiple of 32 in [32, 256] */
  int32_t svd_grad;    /* DCP_SVD_GRAD_* */
  int32_t grid_ctas;   /* CTAs of the grid-update kernels, 0 = default */
  int32_t scatter_mode; /* 0: warp-aggregated scatter, 1: one atomic per particle and node,
                           2: lane pairs with the same base cell merged by one shuffle */
  int32_t min_blocks[3]; /* register-cap levels of k_tri_forward, k_g2p_adj, k_tri_adj: 1 = none,
                           2 = 128, 3 = 96, 4 = 80, 5 = 72, 6 = 64 registers; 0 = default */
  int32_t adj_scatter_mode; /* scatter of the adjoint G2P kernel (k_g2p_adj), same values as
                               scatter_mode, which covers the two P2G kernels */
  int32_t pool_blocks;  /* 0: dense grids (every 4^3-node block of every instance's grid in memory).
                           > 0: paged grids, for large sparse ones: a pool of this many blocks shared
                           by the batch, claimed each substep by the blocks the particles' stencils
                           touch (sparse grid of the reference's grid_v/grid_m, simulation.py:
                           274-302); a substep that needs more sets DCP_STATUS_POOL_FULL */
} DcpOptions;

typedef struct DcpSizes {
  int64_t n_vertex, n_tri, n_operator, n_cube, n_target; /* totals over the batch */
  int64_t state_floats;   /* one state snapshot */
  int64_t rest_floats;    /* rest configuration: D0^-1, n0, x0 */
  int64_t traj_floats;    /* trajectory table */
  int64_t param_floats;   /* parameter table, 8 per instance */
  int64_t static_bytes;   /* device bytes for topology and launch tables */
  int64_t workspace_bytes;/* device scratch bytes (grids, flags, force buffers) */
  int64_t n_tri_chunks, n_point_chunks, total_nodes;
  int64_t grid_blocks;    /* 4^3-node blocks held by each grid array: total_nodes / 64 dense,
                             pool_blocks + 1 (a spare) paged */
} DcpSizes;

typedef struct DcpBatch DcpBatch;

/* Sizes of every buffer of a batch (host only, no CUDA call). */
int dcp_plan(const DcpInstance* inst, int32_t n_inst, const DcpOptions* opt, DcpSizes* out);

/* Builds the launch tables of a batch into `static_dev` and clears
 * `workspace_dev`.  tri_vertices: host, [n_tri_total][3] instance-local vertex
 * ids (lagrangian_mesh_element, taichi_variable_definition.py:29).
 * vertex_rank: host, [n_vertex_total] tie-break order of the Chamfer argmin
 * (NULL = index order).  Replaces the field allocation of
 * taichi_variable_definition.py:1-52. */
int dcp_create(const DcpInstance* inst, int32_t n_inst, const DcpOptions* opt, const int32_t* tri_vertices,
               const int32_t* vertex_rank, void* static_dev, void* workspace_dev, void* stream, DcpBatch** out);
int dcp_destroy(DcpBatch* batch);
int dcp_sizes(const DcpBatch* batch, DcpSizes* out);

/* initialize_ti_field (simulation.py:447-477): rest buffer from the rest
 * positions x0_* ([3][N] each) and the zero state0. */
int dcp_init_state(DcpBatch* batch, const float* x0_vertex, const float* x0_operator, const float* x0_cube,
                   float* state0, float* rest, void* stream);

/* One substep state_in -> state_out: forward(s, grad_update) of
 * simulation.py:480-488 (clear_grid, compute_inplane_F_tmp, inplane_svd, p2g,
 * grid_op, g2p, update_particle_state).  `window` is grad_update. */
int dcp_substep_forward(DcpBatch* batch, const float* params, const float* traj, const float* rest, int32_t step,
                        int32_t window, const float* state_in, float* state_out, void* stream);

/* reset_quadrature_particles (simulation_without_grad.py:471-485) on every
 * cloth: each triangle's rest frame becomes [e1, e2, n] of its current
 * vertices (n: normalised cross product of the eps-normalised edges) and its
 * d3 becomes n.  The reference keeps the stored deformation gradient F, so F - I
 * of the old frame is written to fdev ([9][n_tri] floats) for the stress of
 * the next substep (dcp_replay takes it).  The vertices' rest positions move
 * to their current positions.  Rewrites `rest` and `state` in place. */
int dcp_reset_quadrature(DcpBatch* batch, float* rest, float* state, float* fdev, void* stream);

/* Forward-only replay (the loop of animation(), simulation_without_grad.py:
 * 487-511): n_blocks times, block_steps substeps (step indices first_step,
 * first_step + 1, ...; no window offset) followed by dcp_reset_quadrature.
 * state: in/out; work: a second state buffer; fdev: [9][n_tri] floats.
 * fdev_pending != 0: a reset came before first_step, so its substep takes the
 * stress F from fdev.  After the call fdev is pending when n_blocks > 0. */
int dcp_replay(DcpBatch* batch, const float* params, const float* traj, float* rest, float* state, float* work,
               float* fdev, int32_t first_step, int32_t n_blocks, int32_t block_steps, int32_t fdev_pending,
               void* stream);

/* Reverse of one substep: backward(s, grad_update) of simulation.py:490-506.
 * Given state_in (state s) and adj_out (dL/d state s+1), writes adj_in
 * (dL/d state s) and accumulates grad_params / grad_traj. */
int dcp_substep_backward(DcpBatch* batch, const float* params, const float* traj, const float* rest, int32_t step,
                         int32_t window, const float* state_in, const float* adj_out, float* adj_in,
                         double* grad_params, double* grad_traj, void* stream);

/* compute_loss (parameter_fitting_functions.py:3-15) per instance: one-sided
 * Chamfer sum_q min_p |x_p - t_q|^2 / 3 / Nq on the vertices of `state`.
 * targets: [3][Nq_total]; argmin: [Nq_total] (global vertex index); loss: [n_inst].
 * NaN distances are skipped and set DCP_STATUS_NONFINITE; a target whose
 * distances are all non-finite gets argmin -1 and makes its instance's loss NaN. */
int dcp_chamfer_forward(DcpBatch* batch, const float* rest, const float* state, const float* targets,
                        int32_t* argmin, float* loss, void* stream);
/* compute_loss.grad: adds dL/dx of the vertices into adj_state. */
int dcp_chamfer_backward(DcpBatch* batch, const float* rest, const float* state, const float* targets,
                         const int32_t* argmin, const float* grad_loss, float* adj_state, void* stream);

/* Rollout buffer of dcp_rollout_*: checkpoints every `ckpt_every` substeps plus
 * one recompute segment (floats). */
int64_t dcp_rollout_floats(const DcpBatch* batch, int32_t n_steps, int32_t ckpt_every);
/* Offset (floats) of state `step` inside the rollout buffer after a forward
 * rollout, or -1 when that state is not kept (it lies inside a segment). */
int64_t dcp_rollout_state_offset(const DcpBatch* batch, int32_t n_steps, int32_t ckpt_every, int32_t step);

/* Grid tape (optional; no counterpart in the reference, whose Taichi Tape
 * re-runs P2G inside every adjoint substep): bytes of a tape that keeps, for
 * each of n_steps substeps, the particle-to-grid result (momentum and mass of
 * every active 4^3 node block, plus each vertex's summed corner force) of up to
 * `blocks` active blocks in total.  With a tape, dcp_rollout_forward records
 * and dcp_rollout_backward restores those grids instead of recomputing P2G;
 * substeps that did not fit fall back to recomputing.  A tape belongs to one
 * rollout: pass the same tape, tape_bytes and n_steps to both calls. */
int64_t dcp_tape_bytes(const DcpBatch* batch, int32_t n_steps, int64_t blocks);

/* The Tape-recorded loop of compute_grad (parameter_fitting_functions.py:25-28):
 * n_steps substeps from the state at offset 0 of `buf`, keeping checkpoints.
 * tape: NULL or a grid tape of tape_bytes (dcp_tape_bytes) that this call
 * clears and fills.  use_graph != 0 captures the launches once into a CUDA
 * graph and replays it. */
int dcp_rollout_forward(DcpBatch* batch, const float* params, const float* traj, const float* rest, int32_t window,
                        int32_t n_steps, int32_t ckpt_every, float* buf, void* tape, int64_t tape_bytes,
                        int32_t use_graph, void* stream);

/* The Tape's reverse pass (parameter_fitting_functions.py:25-29 exit): adjoint
 * substeps loss_step-1 .. 0 with segment recompute.  adj_work: [2][state]; slot
 * 0 holds dL/d state(loss_step) on entry; on return dL/d state0 is in slot
 * (loss_step % 2).  tape: NULL or the tape the forward rollout filled. */
int dcp_rollout_backward(DcpBatch* batch, const float* params, const float* traj, const float* rest, int32_t window,
                         int32_t n_steps, int32_t loss_step, int32_t ckpt_every, float* buf, float* adj_work,
                         double* grad_params, double* grad_traj, void* tape, int64_t tape_bytes, int32_t use_graph,
                         void* stream);

/* Kernel launch accounting.  dcp_launch_count: kernels issued on this batch
 * so far (graph replays add the kernels of the captured graph).
 * dcp_profile(1) brackets every subsequent launch with CUDA events on its
 * stream (rollouts then run eagerly); dcp_profile_read fills per-kernel total
 * milliseconds and launch counts, arrays of dcp_kernel_count() entries indexed
 * like dcp_kernel_name(id).  Diagnostics only; no reference counterpart
 * (the reference enables Taichi's kernel profiler, initialization.py:19-20). */
int64_t dcp_launch_count(const DcpBatch* batch);
int dcp_profile(DcpBatch* batch, int32_t enable);
int dcp_profile_read(DcpBatch* batch, double* total_ms, int64_t* launches);
/* Milliseconds of each profiled launch of kernel `id`, in launch order, into
 * ms[0 .. cap); returns the number of such launches (-1 on error). */
int64_t dcp_profile_launches(DcpBatch* batch, int32_t id, double* ms, int64_t cap);
int32_t dcp_kernel_count(void);
const char* dcp_kernel_name(int32_t id);

/* Per-instance DCP_STATUS_* bits (host array of n_inst); synchronises `stream`. */
int dcp_read_status(DcpBatch* batch, int32_t* host_status, int32_t clear, void* stream);

const char* dcp_last_error(void);

/* Chamfer loss of ONE cloth that allocates nothing -- no counterpart in the
 * reference (compute_loss semantics, parameter_fitting_functions.py:3-15).
 * For callers that cannot call cudaMalloc: a plugin whose host application's
 * allocator owns the GPU's memory, or a latency-bound loop in which an
 * allocation is not allowed.  The scratch (per-target minima) is a file-scope
 * device array of DCP_STATIC_MAX_TARGETS floats that every GPU loading the
 * library holds until exit.  The array has one address per CUDA context: the
 * first call in a context (the device's primary context, or a context the
 * caller created with the driver API and made current) looks it up with
 * cudaGetSymbolAddress and caches it under the context's unique id, so make
 * that first call before any stream capture; a context created anew (after
 * cudaDeviceReset, say) is looked up again on its first call.  All calls in a
 * context share the array: calls that overlap on the GPU race.  x0, u (u may
 * be NULL): [3][n_vertex] rest positions and displacements; targets:
 * [3][n_target]; argmin: [n_target] vertex index (first index on ties); loss:
 * one float.  Non-finite distances are skipped; a target whose distances are
 * all non-finite gets argmin -1 and makes the loss NaN.  Returns
 * DCP_ERR_INVALID for n_target > DCP_STATIC_MAX_TARGETS. */
#define DCP_STATIC_MAX_TARGETS (1 << 20)
int dcp_chamfer_forward_static(const float* x0, const float* u, int32_t n_vertex, const float* targets,
                               int32_t n_target, int32_t* argmin, float* loss, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* DIFFCP_B200_H */
