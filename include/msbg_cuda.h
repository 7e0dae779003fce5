/*
 * msbg_cuda.h -- C ABI of the B200 (sm_100a) sparse-grid hot path.
 *
 * Drop-in boundary for the msbg-rs crate's sparse-grid path: the functions
 * below replace, one for one, the crate entry points cited beside each
 * declaration (paths relative to the msbg-rs source tree).  A Rust host binds
 * them with `extern "C"` declarations; the Python package in msbg-rs_b200/
 * binds them with ctypes.
 *
 * Conventions
 *  - Every function returns an int status: MSBG_OK (0) or an MSBG_ERR_* code.
 *    No exception or panic crosses the ABI.  msbg_status_string() names a code;
 *    msbg_last_error() returns the message of the last failure on this thread.
 *  - Handles are opaque.  A context owns one CUDA stream on one device; every
 *    call on objects of a context is ordered on that stream.  Calls are
 *    thread-safe per context object only if the caller serialises them.
 *  - Host-pointer entry points copy their inputs to the device and their
 *    results back (they synchronise the stream before returning).  The
 *    `_device` variants take device pointers, enqueue work and return without
 *    synchronising.
 *  - Block ids (bids) are 64-bit: bid = bx + by*nx + bz*nx*ny
 *    (sparse_grid.rs:157-165); voxel-in-block index vid = x | y<<log2(bsx) |
 *    z<<2*log2(bsx) (sparse_grid.rs:167-175).
 */
#ifndef MSBG_CUDA_H
#define MSBG_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define MSBG_OK 0
#define MSBG_ERR_ARG 1     /* invalid argument (size, id, enum, alignment)  */
#define MSBG_ERR_OOM 2     /* device or host allocation failed              */
#define MSBG_ERR_TIMEOUT 3 /* a bounded device-side wait gave up            */
#define MSBG_ERR_CUDA 4    /* a CUDA runtime call failed                    */
#define MSBG_ERR_STATE 5   /* object used in the wrong state                */
#define MSBG_ERR_NUMERIC 6 /* solver breakdown (NaN / stall)                */

/* ---- enums ----------------------------------------------------------- */
/* Storage element of a grid channel (channel.rs:31-116, stencil.rs:142-192). */
#define MSBG_F32 0  /* f32 payload                                          */
#define MSBG_U16 1  /* `Density`: u16, value = q / 65535, store rounds      */
                    /* half away from zero (stencil.rs:160-174)            */
#define MSBG_BF16 2 /* bf16 payload, store rounds to nearest even           */
#define MSBG_U8 3   /* `Density8`: u8, value = q / 255 (sample.rs:64-70);   */
                    /* writes round(v * 255) (channel.rs:378-382); sweeps  */
                    /* store sqrt-compressed with stochastic rounding      */
                    /* (stencil.rs:176-192)                                */
#define MSBG_F16 4  /* IEEE binary16 payload, store rounds to nearest even  */

/* Stencil of a sweep (solver.rs:44-51). */
#define MSBG_LAPLACIAN 0       /* 7-tap,  laplacian.rs:16-70               */
#define MSBG_MEAN_CURVATURE 1  /* 19-tap, meancurv.rs:17-107               */
#define MSBG_BILAPLACIAN 2     /* 25-tap, bilaplacian.rs:15-97             */

/* Boundary condition (math/boundary.rs:7-16). */
#define MSBG_CLAMP 0
#define MSBG_NEUMANN 1
#define MSBG_DIRICHLET 2

typedef struct msbg_ctx msbg_ctx;
typedef struct msbg_grid msbg_grid;
typedef struct msbg_mac msbg_mac;
typedef struct msbg_poisson msbg_poisson;
typedef struct msbg_unet msbg_unet;
typedef struct msbg_flip msbg_flip;
typedef struct msbg_blockmap msbg_blockmap;

/* ---- context ---------------------------------------------------------- */
const char* msbg_status_string(int status);
const char* msbg_last_error(void);
/* Creates a context on CUDA device `device` with its own stream.
 * (No crate counterpart: the crate runs on the rayon global pool,
 * thread_pool.rs:1-40.) */
int msbg_ctx_create(int device, msbg_ctx** out);
int msbg_ctx_destroy(msbg_ctx* ctx);
int msbg_ctx_synchronize(msbg_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for interop. */
int msbg_ctx_stream(msbg_ctx* ctx, void** stream_out);
/* Number of kernels this library launched on the context since creation. */
int msbg_ctx_kernel_launches(msbg_ctx* ctx, uint64_t* out);
/* Per-kernel timing with CUDA events on the context stream (phase profiling;
 * no crate counterpart beyond MSBG_BUCKET_PROFILE,
 * particles/sort.rs:184-262).  While enabled every kernel launch is bracketed
 * by two events.  The report lists "name launches total_ms" per kernel; it
 * synchronises the stream.  reset != 0 clears the totals after reporting. */
int msbg_ctx_set_timing(msbg_ctx* ctx, int enable);
int msbg_ctx_timing_report(msbg_ctx* ctx, int reset, char* buf, size_t cap, size_t* len_out);
/* Bytes of device scratch currently held by the context's arena. */
int msbg_ctx_scratch_bytes(msbg_ctx* ctx, uint64_t* out);

/* ---- sparse grid (sparse_grid.rs:61-435, blockmap.rs:35-209) ----------- */
/* SparseGrid::new(name, sx, sy, sz, empty_value, full_value, pool)
 * (sparse_grid.rs:109-156).  bsx is a power of two in [1, 32]. */
int msbg_grid_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, int dtype,
                     float empty_value, float full_value, msbg_grid** out);
int msbg_grid_destroy(msbg_grid* grid);
/* out[0..7] = sx, sy, sz, nx, ny, nz, n_blocks, n_value_blocks */
int msbg_grid_dims(const msbg_grid* grid, uint64_t out[8]);
/* ensure_blocks_parallel (sparse_grid.rs:326-355): allocate value blocks for
 * `bids` not yet allocated (a full dummy is replaced), filled with the empty
 * value; existing value blocks are kept. */
int msbg_grid_ensure_blocks(msbg_grid* grid, const uint64_t* bids, size_t n);
/* set_full_block / set_empty_block (sparse_grid.rs:248-262): only for bids
 * that are not value blocks (MSBG_ERR_ARG otherwise). */
/* ensure_blocks_parallel (sparse_grid.rs:326-355) from a device list: the
 * blocks of d_bids (duplicates allowed) that are not value blocks become value
 * blocks holding the empty value; existing blocks keep their data.  Lookups,
 * deduplication and table updates run on the device; only the new ids are
 * read back.  d_slots_out (optional, device, [n]) receives every id's slot. */
int msbg_grid_ensure_blocks_device(msbg_grid* g, const uint64_t* d_bids, size_t n, int32_t* d_slots_out);
int msbg_grid_set_full_blocks(msbg_grid* grid, const uint64_t* bids, size_t n);
int msbg_grid_set_empty_blocks(msbg_grid* grid, const uint64_t* bids, size_t n);
/* set_empty_value / set_full_value (sparse_grid.rs:232-245). */
int msbg_grid_set_values(msbg_grid* grid, float empty_value, float full_value);
/* Ensure + write whole blocks: payload is [n][bsx^3] elements of the grid's
 * dtype (get_block_data_mut + copy). */
int msbg_grid_write_blocks(msbg_grid* grid, const uint64_t* bids, size_t n, const void* payload);
int msbg_grid_write_blocks_device(msbg_grid* grid, const uint64_t* bids, size_t n, const void* d_payload);
/* Read whole blocks (get_value_in_block over the block, sparse_grid.rs:296-305):
 * value blocks give their data, the full dummy its full value, anything else
 * the empty value. */
int msbg_grid_read_blocks(msbg_grid* grid, const uint64_t* bids, size_t n, void* payload);
int msbg_grid_read_blocks_device(msbg_grid* grid, const uint64_t* bids, size_t n, void* d_payload);
/* fill_blocks_parallel (sparse_grid.rs:359-369): fill value blocks among
 * `bids` with `value`; dummies are skipped. */
int msbg_grid_fill_blocks(msbg_grid* grid, const uint64_t* bids, size_t n, float value);
/* Value-block ids in ascending order (active_block_ids, sparse_grid.rs:432).
 * Writes min(count, cap) ids, returns the count in *n_out. */
int msbg_grid_value_block_ids(const msbg_grid* grid, uint64_t* out, size_t cap, size_t* n_out);
/* Device pointer to the payload arena and the slot of each listed bid (-1 if
 * not a value block): zero-copy access for callers that keep data on device. */
int msbg_grid_payload(msbg_grid* grid, void** d_payload, uint64_t* n_slots);
int msbg_grid_slots(const msbg_grid* grid, const uint64_t* bids, size_t n, int32_t* slots_out);

/* ---- halo gather (multires/halo.rs:31-170) ------------------------------ */
/* HaloBlock::fill::<HALO, FULL>(grid, bid, bc) for each listed bid.  out is
 * [n][(bsx+2*halo)^3] f32; halo in {1, 2}.  With full == 0 only the centre,
 * the six faces and the x-edges are written (the rest is 0), as in the
 * reference. */
int msbg_halo_gather(msbg_grid* grid, const uint64_t* bids, size_t n, int halo, int full, int bc,
                     float* out);
int msbg_halo_gather_device(msbg_grid* grid, const uint64_t* d_bids, size_t n, int halo, int full,
                            int bc, float* d_out);

/* ---- 8-colour in-place smoother (solver.rs:141-267) -------------------- */
/* Sweeper::new(grid, ..).sweep(active, stencil, &PdeParams{dt, iterations,
 * do_constr_zero_one}) (solver.rs:154-185) and apply_pde (solver.rs:228-240).
 * Blocks of `active` that are not value blocks are skipped (solver.rs:196-199).
 * The boundary condition is Neumann (solver.rs:205-209).  The plan (colour
 * buckets, neighbour table) is cached per grid and rebuilt only when the
 * active list or the grid's block set changes. */
int msbg_sweep(msbg_grid* grid, const uint64_t* active, size_t n, int stencil, float dt,
               int iterations, int clamp01);
/* The same sweep with the Density8 store's generator made explicit: the
 * store of chunk k (counting every chunk the sweeper stored since it was
 * seeded: sweeps, then colours, then blocks in plan order, then chunks of
 * `lanes` elements in block order) draws from SimdRng::<lanes>::seed(seed)
 * after k + 1 steps (stencil.rs:103-132).  *stream_pos holds k at the first
 * store of this call and is advanced past the last; a fresh sweeper starts at
 * 0.  One rayon thread of the reference (slot 0, seed 0xdeadbeef,
 * solver.rs:109-119) draws exactly this stream.  lanes is the reference
 * build's SIMD width (4, 8 or 16) and must divide the block size.
 * msbg_sweep on a Density8 grid is this call with seed 0xdeadbeef, lanes 16
 * (the block size when that is smaller) and position 0 (apply_pde's fresh
 * sweeper).  Other dtypes ignore the
 * generator (their stores are deterministic) and leave *stream_pos alone. */
int msbg_sweep_stochastic(msbg_grid* grid, const uint64_t* active, size_t n, int stencil, float dt,
                          int iterations, int clamp01, uint32_t seed, int lanes, uint64_t* stream_pos);
/* Multiresolution sweep: the halo of each fine block reads coarser
 * neighbours (levels[b] > levels[bid]) from `coarse` at the fine coordinate
 * >> 1 (fill_multires, multires/halo.rs:187-358); absent blocks read 0.
 * levels is [n_blocks] u8 on the host; coarse.bsx == fine.bsx / 2. */
int msbg_sweep_multires(msbg_grid* fine, msbg_grid* coarse, const uint8_t* levels,
                        const uint64_t* active, size_t n, int stencil, float dt, int iterations,
                        int clamp01);

/* ---- Morton keys and sorts --------------------------------------------- */
/* morton3 (multires/sort.rs:20-22) for n coordinate triples (u64 xyz). */
int msbg_morton3(msbg_ctx* ctx, const uint64_t* xyz, size_t n, uint64_t* keys_out);
/* sort_block_list_morton (multires/sort.rs:35-57): sorts `blocks` in place on
 * the device by the level-scaled Morton key. */
int msbg_sort_block_list_morton(msbg_ctx* ctx, uint64_t* blocks, size_t n, uint64_t nx, uint64_t ny,
                                const uint8_t* levels, size_t n_levels_array, int n_levels);
/* Per-particle Morton sort: key = morton3(trunc(p)) (21 bits per axis), a
 * stable LSD radix sort of (key, index).  keys_out[i] is the i-th smallest key,
 * perm_out[i] the original index of the i-th particle (bit-exact against a
 * stable CPU sort).  pos is [n][3] f32; coordinates must be >= 0 and < 2^21. */
int msbg_morton_sort(msbg_ctx* ctx, const float* pos, size_t n, uint64_t* keys_out, uint32_t* perm_out);
int msbg_morton_sort_device(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys_out,
                            uint32_t* d_perm_out);
/* No counterpart in the reference.  msbg_morton_sort_device without any
 * device allocation, for callers that cannot allocate on the calling path
 * (real-time loops, allocator callbacks, processes whose device memory is
 * reserved up front).  Its temporaries live in a fixed scratch array built
 * into the library (about 5 MB, held by every device that loads the library
 * until exit), so n is limited to 262144 particles; larger n returns
 * MSBG_ERR_ARG.  Each call blocks the host
 * until its stream reaches the end of the sort: it reads the largest key (to
 * choose the number of digit passes) and the bounded-wait status word back,
 * so no call can be captured into a CUDA graph.  Calls share the array, so calls whose GPU work overlaps in time race;
 * calls ordered on one stream do not.  The device address is looked up once
 * per device and kept, so a cudaDeviceReset while the library is loaded is
 * not supported.  Returns MSBG_ERR_STATE while per-kernel timing is enabled
 * (timing creates CUDA events). */
int msbg_morton_sort_noalloc_device(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys_out,
                                    uint32_t* d_perm_out);
/* No counterpart in the reference (test hook).  Runs one radix-sort digit
 * pass whose look-back waits for counts that are never published, with a
 * time limit of limit_ns (1e5 to 1e9): returns MSBG_ERR_TIMEOUT with the
 * context's status word cleared, so the context stays usable. */
int msbg_test_sort_lookback_timeout(msbg_ctx* ctx, uint64_t limit_ns);
/* Applies a sort permutation to per-particle data: dst[i] = src[perm[i]] for
 * items of `width` floats (the payload gather of bucket_particles,
 * fluid/mod.rs:71-91, and bucket_by_block, particles/sort.rs:274-285). */
int msbg_permute_device(msbg_ctx* ctx, const uint32_t* d_perm, size_t n, int width, const float* d_src, float* d_dst);
/* bucket_indices (particles/sort.rs:174-269): block-major permutation of
 * particle block ids.  particle_blocks (capacity n) receives the distinct bids
 * ascending, starts (capacity n + 1) the CSR offsets, perm (n) the particle
 * indices grouped by block; *n_blocks_out the number of distinct blocks.  The
 * order inside a block is the input order (the stable order of the dense
 * counting sort, particles/sort.rs:455-490). */
int msbg_bucket_indices(msbg_ctx* ctx, const uint64_t* bids, size_t n, uint64_t* particle_blocks,
                        uint64_t* starts, uint32_t* perm, size_t* n_blocks_out);
int msbg_bucket_indices_device(msbg_ctx* ctx, const uint64_t* d_bids, size_t n,
                               uint64_t* d_particle_blocks, uint64_t* d_starts, uint32_t* d_perm,
                               size_t* n_blocks_out);

/* ---- staggered MAC grid (fluid/mac.rs) ---------------------------------- */
/* MacGrid::new(sx, sy, sz, pool) (mac.rs:35-45): three face-velocity and three
 * face-mass f32 channels, empty = full = 0. */
int msbg_mac_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, msbg_mac** out);
int msbg_mac_destroy(msbg_mac* mac);
/* Borrowed channel handle: which = 0..2 velocity[X..Z], 3..5 mass[X..Z]. */
int msbg_mac_channel(msbg_mac* mac, int which, msbg_grid** out);
/* MacGrid::zero_blocks (mac.rs:95-102). */
int msbg_mac_zero_blocks(msbg_mac* mac, const uint64_t* bids, size_t n);
/* particles_to_grid (fluid/p2g.rs:141-164): bucket, active_blocks(r_p+1),
 * zero_blocks, splat of mass and momentum to the right faces with
 * w = max(1 - d^2/r_p^2, 0)^3, then normalize_velocity.  pos, vel are [n][3],
 * mass [n] (f32).  Sums are accumulated per particle block in FP64 and
 * combined across blocks in a fixed order: deterministic, no float atomics.
 * bsx is 8 or 16, domain extents are multiples of bsx, 0 < r_p <= 3 and
 * ceil(r_p) <= bsx / 2.
 * *n_active_out (may be NULL) receives the size of the active block set. */
int msbg_p2g(msbg_mac* mac, const float* pos, const float* vel, const float* mass, size_t n, float r_p,
             size_t* n_active_out);
int msbg_p2g_device(msbg_mac* mac, const float* d_pos, const float* d_vel, const float* d_mass, size_t n,
                    float r_p, size_t* n_active_out);
/* particles_to_grid for particles already in Morton order: d_keys are their
 * sorted keys as msbg_morton_sort_device returns them (the caller applied the
 * permutation with msbg_permute_device); the internal sort is skipped.  The
 * result is identical to msbg_p2g_device on the same particles. */
int msbg_p2g_sorted_device(msbg_mac* mac, const float* d_pos, const float* d_vel, const float* d_mass,
                           const uint64_t* d_keys, size_t n, float r_p, size_t* n_active_out);
/* particles_to_grid for particles in the caller's order with the result of a
 * Morton sort of their positions (msbg_morton_sort_device: d_keys sorted,
 * d_perm[i] the caller index of sorted particle i).  The gather into the
 * splat's cell-sorted arrays follows d_perm, so the particle arrays need not
 * be permuted first.  The result is identical to msbg_p2g_device on the same
 * particles (fluid/p2g.rs:141-164 buckets the particles itself). */
int msbg_p2g_permuted_device(msbg_mac* mac, const float* d_pos, const float* d_vel, const float* d_mass,
                             const uint64_t* d_keys, const uint32_t* d_perm, size_t n, float r_p, size_t* n_active_out);
/* Active block set of the last P2G (ascending bids). */
int msbg_mac_active_blocks(const msbg_mac* mac, uint64_t* out, size_t cap, size_t* n_out);
/* MacGrid::normalize_velocity (mac.rs:106-132) over the listed blocks. */
int msbg_mac_normalize_velocity(msbg_mac* mac, const uint64_t* bids, size_t n);
/* MacGrid::divergence (mac.rs:137-171) into `dst` (an f32 grid of the same
 * dims; blocks are ensured). */
int msbg_mac_divergence(msbg_mac* mac, msbg_grid* dst, const uint64_t* active, size_t n);
/* MacSampler::sample::<Linear> (fluid/g2p.rs:15-32): per face component a
 * trilinear cell-centred sample at p - 1/2 e_a (gather_map, math/gather.rs:54-158;
 * trilinear_value, math/sample.rs:203-211).  vel_out is [n][3]. */
int msbg_g2p(msbg_mac* mac, const float* pos, size_t n, int bc, float* vel_out);
int msbg_g2p_device(msbg_mac* mac, const float* d_pos, size_t n, int bc, float* d_vel_out);
/* g2p_blend (fluid/g2p.rs:42-45) on [n][3] arrays. */
int msbg_g2p_blend_device(msbg_ctx* ctx, const float* d_u_old, const float* d_u, const float* d_u_tilde,
                          size_t n, float alpha, float* d_out);
/* msbg_g2p_device followed by msbg_g2p_blend_device in one pass, the
 * samples never stored: d_out[i] = (u_old[i] + (u[i] - u_tilde[i])) alpha +
 * u[i] (1 - alpha) with u the velocity sampled at d_pos[i] (MacSampler::sample,
 * fluid/g2p.rs:26-32; g2p_blend, fluid/g2p.rs:42-45).  d_u_tilde null: u_tilde
 * is the sample itself (the grid unchanged between the two samples).  Bit for
 * bit the two calls' result.  d_out may not alias an input. */
int msbg_g2p_flip_device(msbg_mac* mac, const float* d_pos, size_t n, int bc, const float* d_u_old,
                         const float* d_u_tilde, float alpha, float* d_out);
/* Scalar trilinear Sampler::sample::<Linear> (math/sample.rs:494-512);
 * align 0 = Corner, 1 = CellCentered.  Any storage type: samples are read
 * through Dequant (math/sample.rs:45-70; Density8 linearly, q / 255). */
int msbg_sample_linear(msbg_grid* grid, const float* pos, size_t n, int align, int bc, float* out);
/* Sampler::sample / gradient / hessian (math/sample.rs:493-649) beyond the
 * trilinear value: mode 0 = cubic B-spline value (out[n]), 1 = cubic
 * gradient (out[n][3]), 2 = cubic Hessian (out[n][6]: fxx, fyy, fzz, fxy, fxz,
 * fyz), 3 = trilinear gradient at `align` (out[n][3]).  The cubic basis
 * (math/bspline.rs:4-32) is cell-centred whatever `align` says, with a 4^3
 * window from gather_map (math/gather.rs:54-158); any storage type (read
 * through Dequant as above), blocks >= 4^3. */
int msbg_sample_ext(msbg_grid* grid, const float* pos, size_t n, int mode, int align, int bc, float* out);
int msbg_sample_ext_device(msbg_grid* grid, const float* d_pos, size_t n, int mode, int align, int bc, float* d_out);

/* ---- refinement map (multires/refinement.rs) ---------------------------- */
/* regularize_refinement_map (refinement.rs:63-107): the 2:1 rule on a
 * per-block level map ([nx*ny*nz] u8, 0 = finest), in place; n_levels - 2
 * passes, each moving a block at level >= ll whose finest neighbour (26
 * neighbours) is at ll - 1 up to level ll. */
int msbg_regularize_refinement_map(msbg_ctx* ctx, uint8_t* levels, uint64_t nx, uint64_t ny, uint64_t nz, int n_levels);
int msbg_regularize_refinement_map_device(msbg_ctx* ctx, uint8_t* d_levels, uint64_t nx, uint64_t ny, uint64_t nz,
                                          int n_levels);
/* compute_block_topology (refinement.rs:124-208, levelMg 0): flags_out[bid] =
 * user_flags[bid] (optional) | DOM_BORDER (1 << 1) on the block grid's faces |
 * FINE_COARSE (1 << 3) next to a coarser block | COARSE_FINE (1 << 2) next to
 * a finer one; the FINE_COARSE blocks of level l in block order go to
 * fine_coarse_out + l * n_blocks (optional) and their count to
 * fine_coarse_counts[l]; *n_exists_out counts user EXISTS (1 << 12) blocks. */
int msbg_block_topology(msbg_ctx* ctx, const uint8_t* levels, uint64_t nx, uint64_t ny, uint64_t nz, int n_levels,
                        const uint16_t* user_flags, uint16_t* flags_out, uint64_t* fine_coarse_out,
                        uint64_t* fine_coarse_counts, uint64_t* n_exists_out);

/* ---- BlockMap in device memory (blockmap.rs:35-209) ---------------------- */
/* Open-addressing hash of 64-bit block ids to 32-bit values, probed linearly
 * from (key * 0x9e3779b97f4a7c15) & mask; capacity a power of two >= 4
 * (with_capacity), doubled when live entries plus tombstones would pass 3/4.
 * Keys 2^64 - 1 and 2^64 - 2 are the EMPTY and TOMBSTONE sentinels and are
 * rejected (MSBG_ERR_ARG).  Batches take device arrays. */
int msbg_blockmap_create(msbg_ctx* ctx, uint64_t capacity, msbg_blockmap** out);
int msbg_blockmap_destroy(msbg_blockmap* m);
/* len() and capacity(). */
int msbg_blockmap_len(msbg_blockmap* m, uint64_t* len_out, uint64_t* capacity_out);
/* insert (blockmap.rs:101-127) of n (key, value) pairs; for a key given twice
 * the later value wins, as inserting the batch in order would. */
int msbg_blockmap_insert_device(msbg_blockmap* m, const uint64_t* d_keys, const uint32_t* d_vals, size_t n);
/* update(key, 1, |c| c + 1) (blockmap.rs:153-175) for every key of the batch:
 * the per-key counts of bucket_indices' histogram (particles/sort.rs:174-200). */
int msbg_blockmap_update_add_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n);
/* get (blockmap.rs:86-99): d_out[i] = value of d_keys[i], or `missing`. */
int msbg_blockmap_get_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n, uint32_t missing, uint32_t* d_out);
/* remove (blockmap.rs:129-151): keys become tombstones. */
int msbg_blockmap_remove_device(msbg_blockmap* m, const uint64_t* d_keys, size_t n);
/* sorted_pairs (blockmap.rs:177-187): the live entries by ascending key into
 * device arrays of capacity cap; *n_out = len() (keys_out null: count only). */
int msbg_blockmap_sorted_pairs_device(msbg_blockmap* m, uint64_t* d_keys_out, uint32_t* d_vals_out, size_t cap,
                                      size_t* n_out);

/* ---- surface reconstruction from particles (particles/mod.rs:220-302) ---- */
/* splat (particles/splat.rs:92-319) of device positions d_pos [n][3] into
 * `grid` (Density u16 or f32, empty value 0, full value 1; extents multiples
 * of bsx; r_particle + nb_dist < bsx - 1/2): the footprint blocks of the
 * particles (reach r_scan = r_particle + nb_dist, particles/active.rs:15-47)
 * are allocated and filled with the full value, and every voxel within r_scan
 * of a particle takes the minimum of dist_sq / r_scan^2 (Density: rounded to
 * u16, channel.rs:392-417).  The sorted active bids go to active_out
 * (capacity cap, at least the grid's block count is always enough). */
int msbg_surface_splat_device(msbg_grid* grid, const float* d_pos, size_t n, float r_particle, float nb_dist,
                              uint64_t* active_out, size_t cap, size_t* n_active_out);
/* finalize (particles/finalize.rs:35-71) of the listed value blocks in place:
 * the splatted ratio becomes 1 - clamp(sqrt(ratio) r_scan / (2 r_particle +
 * nb_dist), 0, 1), or 0 where it is >= 0.999 (untouched). */
int msbg_surface_finalize(msbg_grid* grid, const uint64_t* active, size_t n, float r_particle, float nb_dist);
/* reconstruct_and_smooth (particles/mod.rs:279-302) from host positions:
 * splat, finalize, then `iterations` mean-curvature sweeps of step dt with
 * [0, 1] clamping over the active blocks (the PLY loading and placement of the
 * crate's pipeline are left to the caller: see msbg_place_instances). */
int msbg_reconstruct_and_smooth(msbg_grid* grid, const float* pos, size_t n, float r_particle, float nb_dist,
                                int iterations, float dt, uint64_t* active_out, size_t cap, size_t* n_active_out);
/* place (particles/sort.rs:31-144): n_instances copies of the base cloud
 * ([n_base][3], host), instance i at 0.2 smax + 0.6 smax (b_i - bbox_min) /
 * span_max scaled by smin * factor / span_max, kept inside the domain bounds
 * (particles/mod.rs DomainBounds) and the grid; the kept positions go to
 * pos_out ([cap][3], host, instance-major) and their count to *n_out
 * (pos_out null: count only). */
int msbg_place_instances(msbg_ctx* ctx, const float* base, size_t n_base, const float* bbox_min, float span_max,
                         uint64_t sx, uint64_t sy, uint64_t sz, float instance_scale_factor, size_t n_instances,
                         float* pos_out, size_t cap, size_t* n_out);

/* ---- one FLIP transfer step through host arrays ------------------------- */
/* The per-step composition of the crate's transfer entry points that a FLIP
 * loop makes (bucket_particles + particles_to_grid, fluid/p2g.rs:141-164;
 * Sweeper::sweep of the x-face mass, solver.rs:166-185; MacSampler::sample +
 * g2p_blend, fluid/g2p.rs:15-45), with the host<->device copies inside the
 * call.  levels ([n_levels] = one per block of the MAC grid) gives each
 * block's resolution level; `coarse` has half the MAC grid's block size and
 * receives the 2^3 downsample of the x-face mass that feeds the multires
 * halos of the level-0 sweep. */
int msbg_flip_create(msbg_mac* mac, msbg_grid* coarse, const uint8_t* levels, size_t n_levels, msbg_flip** out);
int msbg_flip_destroy(msbg_flip* f);
/* One step: pos, vel ([n][3] f32) and mass ([n]) are copied up; the particles
 * are Morton-sorted (msbg_morton_sort_device), splatted (msbg_p2g_permuted_device,
 * r_p), the x-face mass is smoothed by `sweeps` multires sweeps of `stencil`
 * (dt) over the level-0 blocks of the new active set, velocities are sampled
 * back (Clamp) and blended (alpha), and vel_out[i] ([n][3], host) receives the
 * new velocity of input particle i.  Returns when vel_out is written.  Host
 * arrays from page-locked memory copy at full PCIe speed. */
int msbg_flip_step(msbg_flip* f, const float* pos, const float* vel, const float* mass, size_t n, float r_p, int stencil,
                   float dt, int sweeps, float alpha, float* vel_out);

/* ---- multiresolution transfers (multires/downsample.rs) ----------------- */
/* downsample_channel_avg (downsample.rs:13-59): every value block of `src`
 * (block size b) gets a block in `dst` (block size b/2, same block grid) set
 * to the 2^3 mean. */
int msbg_downsample_avg(msbg_grid* dst, msbg_grid* src);

/* ---- Poisson pressure solve (no crate counterpart) ------------------------
 * The crate's roadmap specifies but does not implement the pressure solve
 * (docs/roadmap.md:608-702): the 7-point operator y = D x - sum_nb x and the
 * relaxation y = w (b + sum_nb x) D^-1 + (1 - w) x, D = 6, zero Dirichlet
 * values outside the active blocks.  Unknowns are the cells of the active
 * blocks in ascending block-id order, [n_active][bsx^3] f32 (the block
 * payload layout).  The multigrid hierarchy halves the block size down to 2,
 * then halves the block grid, down to <= 1024 cells solved by a dense FP64
 * inverse.  Level l rediscretises the 7-point stencil on cells of width 2^l
 * (0.25^l times the stencil, with boundary-corrected diagonals and cell
 * masks); prolongation is cell-centred trilinear and restriction its
 * transpose / 8.  Dot products and norms are FP64. */
int msbg_poisson_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, int bsx, const uint64_t* active,
                        size_t n, msbg_poisson** out);
int msbg_poisson_destroy(msbg_poisson* p);
/* Cells per level (finest first). */
int msbg_poisson_levels(const msbg_poisson* p, uint64_t* cells_out, size_t cap, size_t* n_levels);
/* Pre/post weighted-Jacobi sweeps of the V-cycle and their weight (default 2, 2, 2/3). */
int msbg_poisson_set_smoother(msbg_poisson* p, int nu1, int nu2, float omega);
int msbg_poisson_matvec_device(msbg_poisson* p, const float* d_x, float* d_y);
/* `sweeps` weighted-Jacobi sweeps of A x = b on the finest level, in place. */
int msbg_poisson_jacobi_device(msbg_poisson* p, float* d_x, const float* d_b, float omega, int sweeps);
/* r = b - A x; *norm_out (optional, host) = ||r||_2 in FP64. */
int msbg_poisson_residual_device(msbg_poisson* p, const float* d_x, const float* d_b, float* d_r, double* norm_out);
/* One V-cycle for A x = b, x updated in place. */
int msbg_poisson_vcycle_device(msbg_poisson* p, float* d_x, const float* d_b);
int msbg_poisson_dot_device(msbg_poisson* p, const float* d_a, const float* d_b, double* out);
/* method 0: V-cycles; 1: V-cycle-preconditioned CG.  Iterates from x until
 * ||b - A x|| <= tol ||b|| or max_iter.  history (optional, max_iter entries)
 * receives the relative residual after each iteration. */
int msbg_poisson_solve_device(msbg_poisson* p, int method, float* d_x, const float* d_b, double tol, int max_iter,
                              int* iters_out, double* rel_res_out, double* history);
int msbg_poisson_solve(msbg_poisson* p, int method, float* x, const float* b, double tol, int max_iter,
                       int* iters_out, double* rel_res_out, double* history);
/* Learned preconditioner of methods 2 and 3 (not owned; NULL clears).  The
 * network must be built on the same level-0 blocks (bsx 16) and context.
 * method 2: flexible CG preconditioned by the network followed by a V-cycle
 * on its residual, z = N r + V(r - A N r); method 3: flexible CG
 * preconditioned by V-cycle, network, V-cycle: t = V r + N(r - A V r),
 * z = t + V(r - A t).  Both fall back to the V-cycle (and restart)
 * when the residual stalls for three iterations or a direction loses
 * positivity (method 4, the stationary iteration x += z with the method-3 z,
 * falls back to plain V-cycles when an iteration fails to halve the
 * residual).  msbg_poisson_solve_stats gives, for the last solve (int[4]),
 * V-cycle applications, network applications, the fallback reason (0 none,
 * 1 stall, 2 p.Ap <= 0, 3 r.z <= 0) and the iteration it happened at. */
int msbg_poisson_set_preconditioner(msbg_poisson* p, msbg_unet* net);
/* Method 5: flexible CG whose first |k| preconditioner applications are
 * method 3's (V-cycle, network, V-cycle; without the last V-cycle for k < 0),
 * after which CG restarts from the current iterate with the V-cycle
 * preconditioner; k = 0 makes method 5 plain MG-preconditioned CG.
 * Default 1. */
int msbg_poisson_set_network_lead(msbg_poisson* p, int k);
/* msbg_poisson_solve_device with the solution in FP64 (d_x: initial guess in,
 * solution out).  The f32 entry points round the FP64 solution on return; on
 * smooth right-hand sides that rounding alone can leave a relative residual
 * of order 6 eps / lambda_min (about 1e-5 on thin shells), so callers that
 * need the 1e-6 residual in the stored solution use this one. */
int msbg_poisson_solve_f64_device(msbg_poisson* p, int method, double* d_x, const float* d_b, double tol,
                                  int max_iter, int* iters_out, double* rel_res_out, double* history);
int msbg_poisson_solve_stats(const msbg_poisson* p, int* out);
/* Right-hand side of the learned-preconditioner workload on the device: the
 * divergence of a random smooth velocity field (n_blobs Gaussian blobs,
 * sigma uniform in [4, 16] cells, amplitudes N(0,1)^3, centres in random
 * active blocks) at the level-0 cell centres; `seed` selects the field. */
int msbg_poisson_rhs_device(msbg_poisson* p, uint64_t seed, int n_blobs, float* d_b);
/* Trains the network on pairs the solver generates: per right-hand side
 * (seeds seed*1000003 + i), the MG-PCG solution x* to 1e-7, then plain
 * V-cycles from zero giving (residual r_k, error x* - x_k) after each cycle
 * (target 0), or (r_k - A V r_k, x* - x_k - V r_k) (target 1, for method 3).
 * target | 2 takes the pairs along MG-preconditioned CG iterates instead of
 * plain V-cycles.  Pairs fill a device pool of `pool` slots; after each right-hand side,
 * steps_per_rhs Adam steps (learning rate lr) on random pool slots.  The
 * network's output scale is set from the first right-hand side's pairs.
 * loss_hist (may be NULL) receives up to hist_cap per-step losses. */
int msbg_poisson_train_preconditioner(msbg_poisson* p, int n_rhs, int mg_iters, int steps_per_rhs, int pool, float lr,
                                      int target, uint64_t seed, double* loss_hist, int64_t hist_cap,
                                      int64_t* steps_out);
/* Mean relative L2 errors over fresh pairs (as above, seeds from `seed`):
 * out[0] network alone ||N r - e|| / ||e||, out[1] one V-cycle
 * ||V r - e|| / ||e||, out[2] V-cycle plus network correction. */
int msbg_poisson_eval_preconditioner(msbg_poisson* p, int n_rhs, int mg_iters, uint64_t seed, double* out3);

/* ---- block-sparse 3x3x3 convolution on the tensor cores ------------------
 * No counterpart in the reference (the learned preconditioner of the pressure
 * solve).  A level's feature map is bf16 [cells][C], cells in block order
 * (block k = cells k*bs^3 .. (k+1)*bs^3-1, payload order), zero outside the
 * active blocks; nbr27 is int32 [n_blocks][27] (slot of neighbour block
 * (dx,dy,dz) at (dx+1)+3(dy+1)+9(dz+1), -1 if absent).  Weights are bf16
 * [27][cout][cin]; cin, cout in {16, 32, 64}; lg = log2(bs) in [1, 5].
 * msbg_conv3_forward_device: y = relu?(conv(x) + bias), y bf16 or f32
 * (out_f32) [cells][cout]; bias f32 [cout] or NULL.
 * msbg_conv3_wgrad_device: dw = sum_c x[c + d(t)] dy[c]^T, f32 [27][cout][cin].
 * Both synchronise and return MSBG_ERR_TIMEOUT if a bounded wait gave up. */
int msbg_conv3_forward_device(msbg_ctx* ctx, const int32_t* d_nbr27, int64_t n_blocks, int lg, int cin, int cout,
                              const uint16_t* d_x, const uint16_t* d_w, const float* d_bias, int relu, int out_f32,
                              void* d_y);
int msbg_conv3_wgrad_device(msbg_ctx* ctx, const int32_t* d_nbr27, int64_t n_blocks, int lg, int cin, int cout,
                            const uint16_t* d_x, const uint16_t* d_dy, float* d_dw);

/* ---- learned preconditioner: block-sparse 3D U-Net ------------------------
 * No counterpart in the reference.  Three levels on the same blocks (16^3,
 * 8^3, 4^3 cells), 16/32/64 channels, 3x3x3 convolutions with bf16 weights
 * and activations and f32 accumulation on the tensor cores; forward and
 * backward run on the device, Adam updates f32 master weights.  The network
 * acts on level-0 vectors of a Poisson solve (f32 [n_blocks][4096], blocks
 * in ascending id order): z = rms(r) * out_scale * N(r / rms(r)).
 * Parameters are one flat f32 array; msbg_unet_layers lists per layer
 * (level, cin, cout, cin_real, cout_real, relu, w_offset, b_offset), weights
 * [27][cout][cin] (padded channels stay zero).  A train step returns the loss
 * sum((out_scale y - e/rms(r))^2) / sum((e/rms(r))^2) and leaves the
 * gradient readable with msbg_unet_get_grads; update != 0 applies Adam. */
int msbg_unet_create(msbg_ctx* ctx, uint64_t sx, uint64_t sy, uint64_t sz, const uint64_t* active, size_t n,
                     uint64_t seed, msbg_unet** out);
int msbg_unet_destroy(msbg_unet* net);
int msbg_unet_num_params(const msbg_unet* net, size_t* out);
int msbg_unet_layers(const msbg_unet* net, int64_t* out, size_t cap, size_t* n_out);
int msbg_unet_get_params(msbg_unet* net, float* out);
int msbg_unet_set_params(msbg_unet* net, const float* in);
int msbg_unet_get_grads(msbg_unet* net, float* out);
int msbg_unet_set_output_scale(msbg_unet* net, float s);
int msbg_unet_apply_device(msbg_unet* net, const float* d_r, float* d_z);
int msbg_unet_forward_raw_device(msbg_unet* net, const float* d_r, float* d_y);
int msbg_unet_train_step_device(msbg_unet* net, const float* d_r, const float* d_e, float lr, int update,
                                double* loss_out);

/* ---- batched Poisson solves ------------------------------------------------
 * No counterpart in the reference.  Many independent problems (each a domain
 * dims[3p..3p+2], block size bsx[p] in {4..32}, active block ids active[p]
 * [n_active[p]]) are stacked in one hierarchy per block size (problems never
 * touch at any level).  Problem p's level-0 cells are a contiguous range of
 * its group's vectors (msbg_batch_problem), blocks in ascending id order.
 * msbg_batch_buffers gives the group's device right-hand side (f32) and
 * solution (FP64).  tune != 0 autotunes every level but the coarsest: the
 * z-planes per CTA (2, 4, 8 or 16) of the 16^3 tile kernel on levels of whole
 * 16^3 blocks, the launch shapes (threads, CTAs per SM) of the Jacobi and
 * residual kernels elsewhere (msbg_batch_tuning: per level cfg_out[3l..3l+2]
 * = Jacobi shape index, residual shape index, tile z-planes or 0, and the
 * level's cells; cap counts levels).  msbg_batch_solve runs
 * MG-preconditioned CG with per-problem scalars on the device.  A cycle is
 * iters_per_cycle iterations over all problems plus the FP64 residual
 * replacement; the whole solve is a single CUDA graph launch whose
 * device-side while loop (a conditional graph node) runs cycles until every
 * problem reaches relative residual tol (true residual of the FP64 solution)
 * or max_cycles have run; the host waits once, at the end.  iters_out and
 * rel_out are per problem, cycles_out the cycles the loop ran.
 * msbg_poisson_autotune tunes a single solve's hierarchy the same way
 * (cfg_out as above; cap counts ints). */
typedef struct msbg_batch msbg_batch;
int msbg_batch_create(msbg_ctx* ctx, int n_problems, const int* bsx, const uint64_t* dims, const uint64_t* const* active,
                      const size_t* n_active, int tune, msbg_batch** out);
int msbg_batch_destroy(msbg_batch* batch);
int msbg_batch_groups(const msbg_batch* batch, int* n_groups);
int msbg_batch_problem(const msbg_batch* batch, int p, int* group, uint64_t* cell_offset, uint64_t* n_cells);
int msbg_batch_buffers(msbg_batch* batch, int group, float** d_b, double** d_x, uint64_t* n_cells, int* bsx);
/* Host copies of one problem's right-hand side (f32, in) and solution (FP64, out). */
int msbg_batch_set_rhs(msbg_batch* batch, int p, const float* b);
int msbg_batch_get_solution(msbg_batch* batch, int p, double* x);
int msbg_batch_tuning(const msbg_batch* batch, int group, int* cfg_out, uint64_t* cells_out, size_t cap,
                      size_t* n_levels);
int msbg_batch_solve(msbg_batch* batch, double tol, int iters_per_cycle, int max_cycles, int zero_x, int* iters_out,
                     double* rel_out, int* cycles_out);
int msbg_poisson_autotune(msbg_poisson* p, int* cfg_out, size_t cap, size_t* n_levels);
/* Sets the first n_levels levels' choices (cfg as msbg_poisson_autotune
 * writes it: Jacobi shape, residual shape, tile per level), e.g. a tuning
 * saved from an earlier run.  Tile 1 is the quad tile (one 64-thread CTA per
 * 16^3 block, four cells per thread), 2/4/8/16 the slab tile with that many
 * z-planes per 256-thread CTA; every choice computes the same bits. */
int msbg_poisson_set_tuning(msbg_poisson* p, const int* cfg, size_t n_levels);

#ifdef __cplusplus
}
#endif
#endif /* MSBG_CUDA_H */
