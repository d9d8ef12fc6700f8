/*
 * psb200.h — C ABI of the B200 placement-search engine for spectral 3D packing.
 *
 * Every entry point takes plain host pointers and sizes, returns an int status
 * (PSB_OK == 0) and never throws.  On failure psb_last_error() gives a message.
 * Voxel grids are int32, row-major, element (i,j,k) at [(i*ny + j)*nz + k]
 * (the reference's FlatVoxelGrid layout, spectral_packing/types.h:24-38).
 *
 * Each function below names the reference symbol it replaces.  The pybind11
 * module psacking_b200._core binds them under the reference's Python names
 * (spectral_packing/bindings.cpp:654-930).
 */
#ifndef PSB200_H
#define PSB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PSB_OK            0
#define PSB_ERR_ARG       1  /* bad shape, size or pointer                     */
#define PSB_ERR_CUDA      2  /* a CUDA runtime call failed (message has it)    */
#define PSB_ERR_STATE     3  /* context missing / not initialised             */
#define PSB_ERR_OVERLAP   4  /* place_in_tray: item intersects tray contents   */
#define PSB_ERR_LIMIT     5  /* a device-side iteration or capacity limit hit  */
#define PSB_ERR_NODEVICE  6  /* no CUDA device visible                         */

/* ---- search modes -------------------------------------------------------
 * PSB_MODE_SCAN : the single-call CPU-scored search, packing.cpp:590-642.
 *   score = prox + 1e8*pow(k/nz, 3); ties -> lowest linear index;
 *   found iff best < 1e9 (constants.h INF).
 * PSB_MODE_BLOCK: the GPU-context search, fft3.cu:147-175 + 527-563 + 1330-1372.
 *   score = fma((1e8*qz)*qz, qz, prox), qz = k/nz; ties -> lowest 256-block,
 *   then lowest bit-reversed 8-bit offset inside the block; found iff < 1e29.
 * PSB_FLAG_INTERLOCK: only positions reachable from the exit faces by the
 *   Algorithm-3 flood fill count (fft3.cu:234-455, 1377-1459).            */
#define PSB_MODE_SCAN      0
#define PSB_MODE_BLOCK     1
#define PSB_FLAG_INTERLOCK 0x10

/* diagnostic bits in psb_result.diag */
#define PSB_DIAG_EXACT_RESCORE   0x1  /* FP32 error bound >= 0.5: candidates re-scored exactly */
#define PSB_DIAG_AMBIGUOUS_COLL  0x2  /* a collision value fell near a rounding boundary      */
#define PSB_DIAG_FALSE_FREE      0x4  /* exact re-check rejected an FP32 "free" candidate      */
#define PSB_DIAG_BOUND_EXCEEDED  0x8  /* observed FP32 error exceeded half the error bound     */
#define PSB_DIAG_CAND_OVERFLOW   0x100 /* tie-guard candidates exceeded the list capacity     */
#define PSB_DIAG_SKIPPED         0x200 /* orientation larger than the tray, not searched      */
#define PSB_DIAG_FLOOD_FILL      0x400 /* interlocking search: the winner over the free cells
                                          had no straight free run to a seed face, so the
                                          flood fill and a second selection ran             */
#define PSB_DIAG_DIRECT          0x800 /* few candidates left by the pre-filter: decided by direct
                                          exact checks and exact proximity sums, no transforms */
#define PSB_DIAG_LATE_DIRECT    0x1000 /* few ok cells left after the collision pass: their proximity
                                          by exact sums, no proximity transform                 */

typedef struct psb_result {
    int32_t x, y, z;       /* placement of the item array origin, or -1,-1,-1      */
    int32_t found;         /* 1 when a valid placement exists                       */
    double  score;         /* reference score of the placement (0.0 when not found) */
    int32_t orientation;   /* index into the orientation list, -1 when not found    */
    uint32_t diag;         /* PSB_DIAG_* bits                                       */
    int32_t n_candidates;  /* candidates examined by the exact tie guard             */
    float   err_ratio;     /* largest |FP32 - exact| / bound among re-scored candidates */
} psb_result;

typedef struct psb_tray psb_tray;   /* a device-resident tray (GPUTrayContext) */

/* ---- library (no counterpart in the reference: its pybind11 module prints
 *      CUDA errors, fft3.cu:59-91, and raises Python exceptions) --------- */
const char* psb_version(void);
/* Copies the calling thread's last error message into buf (NUL-terminated). */
int psb_last_error(char* buf, size_t len);
/* Number of visible CUDA devices (0 without a GPU; never an error). */
int psb_device_count(int* n);

/* ---- stateless reference entry points ---------------------------------- */

/* dft_conv3 (fft3.cu:643-715 / packing.cpp:162-213): linear 3-D convolution of
 * two same-shape grids, truncated to that shape, rounded to int32. */
int psb_dft_conv3(const int32_t* a, const int32_t* b, int nx, int ny, int nz, int32_t* out);

/* dft_corr3 (packing.cpp:215-229): out[t] = sum_x b[x] * a[t+x], a zero outside. */
int psb_dft_corr3(const int32_t* a, const int32_t* b, int nx, int ny, int nz, int32_t* out);

/* dft_corr3 for callers that cannot allocate device memory.  No counterpart
 * in the reference.  Some callers own every byte of device memory themselves
 * (a framework's caching allocator, a fixed memory budget) or must not call
 * cudaMalloc/cudaFree because those calls synchronise the device and are not
 * stream-ordered (latency-critical loops next to other work on the GPU).
 * This variant computes exactly what psb_dft_corr3 computes, but:
 *   - d_a, d_b and d_out are DEVICE pointers to (nx,ny,nz) int32 grids that
 *     the caller provides; all work, including writing the transform
 *     descriptors and twiddle tables, is queued on `stream` (a cudaStream_t,
 *     NULL for the default stream) and the call returns without waiting for
 *     the GPU;
 *   - its scratch is a fixed 3 MiB array in the library's device code, held
 *     by every GPU that loads the library until the process exits;
 *   - every axis must be <= 32 voxels; larger grids return PSB_ERR_LIMIT;
 *   - it calls no cudaMalloc/cudaFree or other allocating routine.
 * The first call on each device looks up the array's device address and
 * keeps it (make that first call before any stream capture; the address is
 * not looked up again, so do not use the function across a
 * cudaDeviceReset).  All calls share the one array: calls that overlap on
 * the GPU (different streams, or different host threads) race and must be
 * serialised by the caller; calls queued on one stream are safe.  Nothing in
 * the array needs to start at zero: each call writes all it reads. */
int psb_dft_corr3_noalloc(const int32_t* d_a, const int32_t* d_b, int nx, int ny, int nz,
                          int32_t* d_out, void* stream);

/* collision_grid (packing.cpp:241-252, binding bindings.cpp:360-372): the item
 * is zero-padded to the tray shape; out = dft_corr3(tray, item) with positions
 * where the item would leave the tray raised to at least 1. */
int psb_collision_grid(const int32_t* tray, int nx, int ny, int nz,
                       const int32_t* item, int ex, int ey, int ez, int32_t* out);

/* calculate_distance (fft3.cu:944-1004): L1 distance to voxels equal to 1;
 * nx+ny+nz+10 everywhere when there is none. */
int psb_calculate_distance(const int32_t* grid, int nx, int ny, int nz, int32_t* out);

/* interlocking_free_positions (bindings.cpp:561-648 + fft3.cu:348-402):
 * 1 where the object can be placed and slid out of the tray, else 0. */
int psb_interlocking_free_positions(const int32_t* tray, int nx, int ny, int nz,
                                    const int32_t* obj, int ex, int ey, int ez,
                                    int32_t* out);

/* fft_search_placement (packing.cpp:590-642, binding bindings.cpp:182-203):
 * distance field from the tray, then a PSB_MODE_SCAN search. */
int psb_fft_search_placement(const int32_t* item, int ex, int ey, int ez,
                             const int32_t* tray, int nx, int ny, int nz,
                             psb_result* out);

/* place_in_tray (packing.cpp:773-788, binding bindings.cpp:259-276): out_tray
 * receives a copy of tray with item voxels (>0) written as item_id at pos.
 * PSB_ERR_OVERLAP when an item voxel meets an occupied voxel; overlap_ijk
 * (may be NULL) then gets the first such tray cell in row-major order. */
int psb_place_in_tray(const int32_t* item, int ex, int ey, int ez,
                      const int32_t* tray, int nx, int ny, int nz,
                      int px, int py, int pz, int32_t item_id,
                      int32_t* out_tray, int32_t* overlap_ijk);

/* ---- device-resident tray (GPUTrayContext, fft3.cu:1040-1502) ----------- */

int psb_tray_create(int nx, int ny, int nz, psb_tray** out);
int psb_tray_destroy(psb_tray* t);
int psb_tray_dims(const psb_tray* t, int* nx, int* ny, int* nz);

/* gpu_tray_context_init (fft3.cu:1106-1175): upload the tray and its distance
 * field and build both spectra.  phi == NULL computes the distance field on
 * the device from the tray. */
int psb_tray_set(psb_tray* t, const int32_t* tray, const int32_t* phi);

/* Copy the device tray / distance field back to the host. */
int psb_tray_get(psb_tray* t, int32_t* tray, int32_t* phi);

/* Statistics of the device tray for the packing result
 * (BinPacker._calculate_stats, packer.py:582-601): the number of cells > 0
 * and their bounding box lo[3]..hi[3] (inclusive; -1 when none), computed
 * on the device instead of over a host copy. */
int psb_tray_stats(psb_tray* t, long long* occupied, int32_t* lo, int32_t* hi);

/* fft_search_batch / fft_search_batch_interlocking_free / gpu_tray_search
 * (fft3.cu:1506-1632): search n orientation arrays against the tray.
 * items[o] points at an (dims[3o],dims[3o+1],dims[3o+2]) grid.  Orientations
 * larger than the tray are skipped.  per_orient (may be NULL) receives each
 * orientation's own best; out receives the best over orientations (strict <,
 * first wins) with out->orientation its index. */
int psb_tray_search(psb_tray* t, const int32_t* const* items, const int32_t* dims,
                    int n, int mode_flags, psb_result* out, psb_result* per_orient);

/* Device-side place (packing.cpp:773-788) on the resident tray, followed by the
 * spectrum update (and the distance-field update when a voxel equal to 1 was
 * written).  Rejects overlaps with PSB_ERR_OVERLAP and leaves the tray intact. */
int psb_tray_place(psb_tray* t, const int32_t* item, int ex, int ey, int ez,
                   int px, int py, int pz, int32_t item_id);

/* ---- device-resident greedy packing loop (BinPacker.pack_voxels,
 *      spectral_packer/packer.py:366-544) ------------------------------------
 * items are already in packing order.  Orientations are generated on the
 * device from each item by the signed axis permutations in orient_maps
 * (n_orient entries of 6 ints: src_axis[3], flip[3]), which the caller derives
 * from its orientation function.  Mode selection follows packer.py:
 * interlock != 0 -> batch interlocking-free search (PSB_MODE_BLOCK);
 * n_orient > 1   -> per-orientation cached search (PSB_MODE_BLOCK);
 * otherwise      -> fft_search_placement (PSB_MODE_SCAN).
 * out_placements gets one psb_result per item (orientation = index into the
 * orientation list).  Item k is written with id_offset + (number placed
 * before it) + 1.  The final tray is copied to final_tray when not NULL. */
int psb_pack(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n_items,
             const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
             psb_result* out_placements, int32_t* final_tray);

/* psb_pack split in two (the same loop, packer.py:447-528): stage the items
 * of a run on the device once (their
 * runs, bounds and filter samples are computed here), then run the greedy
 * loop over the staged items.  psb_pack gives the same results as
 * psb_pack_stage + psb_pack_staged; with 64 items or more it stages the
 * items after the first 32 while those are searched. */
int psb_pack_stage(psb_tray* t, const int32_t* const* items, const int32_t* dims, int n_items);
int psb_pack_staged(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                    psb_result* out_placements, int32_t* final_tray);

/* ---- orientation-sharded packing loop over several GPUs ------------------
 * The greedy loop of psb_pack_staged with one tray's orientations spread
 * over `world` ranks (one process and GPU each, every rank holding the whole
 * tray): rank r searches the orientations o with o % world == r.  Per item,
 * the rank's best (PSB_SHARD_RECORD_BYTES, with the global orientation
 * index) is written to the device buffer d_local on the tray's stream
 * (psb_tray_stream); then exchange(ctx) is called on the host, once per item
 * in item order, and must queue on that stream the gathering of every rank's
 * record into d_all (world records in rank order, e.g. an NCCL all-gather)
 * and return 0.  The merged winner -- the smallest score, on equal scores the
 * lowest orientation index, the reference's strict < over orientations
 * (spectral_packing/fft3.cu:1625, spectral_packer/packer.py:500) -- is placed
 * on every rank, so the trays stay identical without being exchanged and the
 * results equal psb_pack_staged's.  world == 1 needs no exchange (NULL): the
 * record is copied to d_all.  The reference packs on one GPU only; this
 * entry point has no counterpart there. */
#define PSB_SHARD_RECORD_BYTES 32
typedef int (*psb_exchange_fn)(void* ctx);
int psb_pack_staged_sharded(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock, int32_t id_offset,
                            int rank, int world, void* d_local, void* d_all, psb_exchange_fn exchange, void* ctx,
                            psb_result* out_placements, int32_t* final_tray);

/* ---- detailed packing run and the learned orientation proposal ---------
 * None of these has a counterpart in the reference: the learned-proposal
 * form of the placement search (a small 3-D CNN that ranks an item's 24
 * orientations so that only the best k are searched exactly) is an addition
 * of this engine, described in psb_proposal.cuh.                          */

/* psb_pack_staged, also returning every orientation's own result
 * (per_orient: n_items x n_orient, may be NULL) and the 32x32 pooled height
 * map of the tray before each item (hmaps: n_items x 1024 floats, may be
 * NULL): the plain method's training data for the proposal network.       */
int psb_pack_staged_detail(psb_tray* t, const int32_t* orient_maps, int n_orient, int interlock,
                           int32_t id_offset, psb_result* out_placements, int32_t* final_tray,
                           psb_result* per_orient, float* hmaps);

/* ---- learned orientation proposal (no counterpart in the reference) ---- */
typedef struct psb_proposal psb_proposal;   /* network weights and work buffers on one GPU */
int psb_prop_create(psb_proposal** out);
int psb_prop_destroy(psb_proposal* p);
int psb_prop_num_params(size_t* n);
/* Host FP32 parameter vector in the layer order of the network; weights are
 * used as BF16 (round to nearest even), biases as FP32.  Resets Adam.     */
int psb_prop_set_params(psb_proposal* p, const float* params, size_t n);
int psb_prop_get_params(psb_proposal* p, float* params, size_t n);
/* Forward pass over n_items items of 24 orientations each: d_grids
 * [n_items*24][32^3], d_hmaps [n_items][1024] (device).  With d_target
 * (soft targets [n_items][24]) and d_mask ([n_items][24], 1 = the
 * orientation fits the tray): the masked softmax cross-entropy (h_loss)
 * and every parameter's gradient (psb_prop_get_grads).  d_logits
 * [n_items*24] may be NULL.                                               */
int psb_prop_forward_backward(psb_proposal* p, const float* d_grids, const float* d_hmaps, const float* d_mask,
                              const float* d_target, int n_items, float* d_logits, float* h_loss);
int psb_prop_get_grads(psb_proposal* p, float* grads, size_t n);
/* One Adam step on the last gradients. */
int psb_prop_adam_step(psb_proposal* p, float lr, float beta1, float beta2, float eps);
/* The network's item inputs: per item (host int32 arrays), its occupancy
 * scaled into a 32^3 grid (s = ceil(max extent / 32), a cell holds the
 * occupied fraction of its s^3 block), turned by each orientation map
 * (src_axis[3], flip[3]) -> d_out [n_items][n_orient][32^3] (device).     */
int psb_prop_item_grids(const int32_t* const* items, const int32_t* dims, int n_items,
                        const int32_t* orient_maps, int n_orient, float* d_out);
/* The network's tray input: per column 1 + highest occupied z (0 when empty)
 * over nz, averaged over ceil(nx/32) x ceil(ny/32) blocks -> d_out [32*32]. */
int psb_height_map(const int32_t* d_tray, int nx, int ny, int nz, float* d_out);
/* The packing loop of psb_pack_staged with the proposal: before each item's
 * search the network ranks its 24 orientations (orient_maps must be the 24
 * of get_24_orientations) and only the top-k are searched, or all of them
 * when the top-k softmax mass is below `margin`.  gate_stats (may be NULL)
 * receives [items gated, full-sweep fallbacks].                           */
int psb_pack_staged_prop(psb_tray* t, psb_proposal* prop, const int32_t* orient_maps, int n_orient, int interlock,
                         int32_t id_offset, int topk, float margin, psb_result* out_placements,
                         int32_t* final_tray, int32_t* gate_stats);

/* ---- mesh voxelizer (voxelize_stl) --------------------------------------
 * Replaces spectral_packing/bindings.cpp:285-302 (py_voxelize_stl) and
 * packing.cpp:540-588 (voxelize): exact vertex merge, the box transform to
 * `resolution` voxels along the longest side (5% margin, 16-bit fixed
 * point), rasterization along the three axes with the parity bit per axis,
 * surface voxels only (the reference compiles the inside fill out), tight
 * bounding box.  tris: ntri x 3 vertices x (x, y, z) floats, as read from an
 * STL file.  out must hold resolution^3 int32; it receives the tight grid
 * (C order, values 0/1) and dims_out its shape ({0,0,0} when empty).  The
 * triangle degeneracy test is evaluated modulo 2^32, as the reference's
 * 32-bit int products wrap (packing.cpp rasterize).                        */
int psb_voxelize_mesh(const float* tris, int ntri, int resolution, int32_t* out, int32_t* dims_out);

/* ---- engine settings (no counterpart in the reference) ------------------
 * Kernel variant switch (default on): FFT lengths 64, 100, 128, 240 use
 * the specialised two-pass kernels; off forces the generic mixed-radix path
 * (used by the tests to check both). */
int psb_set_fast_fft(int on);
/* Plane-pass kernel for the specialised FFT lengths: 3 (default; warp-owned
 * line transforms, two block barriers per field) or 2 (every radix pass
 * spread over the CTA).  Same results; a tuning and comparison switch.
 * No counterpart in the reference (cuFFT there). */
int psb_set_plane_variant(int v);
/* Candidate pre-filter of the packing loop (psb_pack*, default on): before
 * an item's collision transforms, a bit-parallel test of up to 128 of its
 * voxels against the tray proves most translations (and often whole
 * orientations or x planes) blocked; those are skipped, every other cell is
 * decided exactly as before.  It starts once the tray's occupied cells plus
 * the items searched so far reach a quarter of the tray (before that it
 * rarely rules anything out).  Same placements either way; the switch exists
 * for comparisons.  No counterpart in the reference. */
int psb_set_cand_filter(int on);
/* Orientations the pre-filter leaves with at most n candidate translations
 * (default 4096; 0 disables) skip the transforms: each candidate is checked
 * exactly against the item's voxel columns and the free ones are scored by
 * exact integer proximity sums.  Same placements either way. */
int psb_set_direct_max(int n);
/* Pre-filter cut-off: a group of 32 translations stops testing samples when,
 * after 32 samples, more than pct % of them still pass (open space, nothing
 * to skip there); default 50, 0 tests every sample.  Any subset of samples
 * keeps the filter exact, so results never depend on it. */
int psb_set_filter_cut(int pct);
/* Orientations left with at most n ok cells (free, or reachable in the
 * interlocking mode) after the collision pass skip the proximity transforms:
 * those cells are scored by exact integer proximity sums over the item's
 * z-runs instead (default 0: off, measured neutral on the benchmark).  Same
 * placements either way.
 * No counterpart in the reference. */
int psb_set_late_direct_max(int n);
/* Bound on the flood fill's union-find work per run lookup or merge
 * (retries and path steps).  Past it the kernels stop following the chain,
 * every access staying in bounds, and the search returns PSB_ERR_LIMIT
 * instead of an answer.  n <= 0 restores the default (2^22, far above any
 * chain a tray of 2^31 cells can form with path halving).  The reference
 * bounds its flood fill by nx+ny+nz propagation sweeps instead
 * (fft3.cu:437); this bound exists so that no device loop can spin. */
int psb_set_uf_limit(int n);
/* Test hooks, no counterpart in the reference: psb_debug_fail_alloc(n)
 * makes the n-th device allocation of the engine from now on fail as a
 * CUDA allocation error would (PSB_ERR_CUDA); 0 disarms it.
 * psb_debug_live_allocs reports the engine's device allocations not yet
 * freed, so a test can check that a failed call freed what it allocated. */
int psb_debug_fail_alloc(int n);
int psb_debug_live_allocs(long long* n);
/* The 24 orientations are 6 axis permutations x 4 flip patterns.  On: the
 * z,y transforms of each permutation run once per item and the x pass reads
 * every flip from them (row reversal, column map, conjugation, phase).  Off
 * (the default, faster on B200): every orientation is transformed on its
 * own.  Same results; a comparison switch.  No counterpart in the
 * reference. */
int psb_set_share_flips(int on);

/* Many independent trays (the many-tray form of the benchmark set; no
 * counterpart in the reference, which packs one tray per call): tray i
 * has dims tray_dims[3i..3i+2] and items_per_tray[i] items, which follow the
 * previous trays' items in `items` / `item_dims` and are already in packing
 * order.  Each tray starts empty and is packed exactly as psb_pack would;
 * up to `concurrency` trays run at once, each on its own CUDA stream and host
 * worker thread.  out_placements has one result per item (same order);
 * final_trays (may be NULL) has one output grid per tray. */
int psb_pack_many(int n_trays, const int32_t* tray_dims, const int32_t* const* items, const int32_t* item_dims,
                  const int32_t* items_per_tray, const int32_t* orient_maps, int n_orient, int interlock,
                  int concurrency, psb_result* out_placements, int32_t* const* final_trays);

/* ---- tracing (the reference's SCOPED_TIMER, spectral_packing/timing.h:11-31,
 *      as CUDA events around every kernel launch; off by default) ---------- */
int psb_profile_enable(int on);          /* clears previous records            */
/* "name launches total_ms" lines, one per kernel, after synchronising. */
/* Restrict the profiler to the named kernels (comma-separated profiler
 * names, e.g. "k_plane,k_xpass"); NULL or "" records every kernel. */
int psb_profile_filter(const char* names);
int psb_profile_report(char* buf, size_t len);
/* ---- tray introspection for the benchmark (no counterpart in the reference)
 * FFT grid of a tray (F[0..2] >= nx, ny, nz; 2^a 3^b 5^c 7^d). */
int psb_tray_fft_dims(const psb_tray* t, int* F);
/* The CUDA stream (cudaStream_t) a tray's kernels run on. */
int psb_tray_stream(psb_tray* t, void** stream);
/* Work counters of a tray's transform kernels since the last reset (the
 * measurement's algorithmic bytes): out[0] collision x-pass orientations,
 * out[1] the sum of their item x extents, out[2] their stored product planes,
 * out[3] collision plane-pass planes, out[4] their row pairs, out[5]
 * proximity x-pass orientations, out[6] their stored planes (also the
 * proximity plane-pass planes), out[7] proximity plane-pass row pairs.
 * out may be NULL; reset != 0 zeroes them after the copy. */
int psb_tray_work(psb_tray* t, unsigned long long* out, int reset);

#ifdef __cplusplus
}
#endif
#endif /* PSB200_H */
