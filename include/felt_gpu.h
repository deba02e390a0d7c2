/* felt_gpu.h - C ABI of the B200 (sm_100a) sparse-field level-set engine.
 *
 * This is the thin boundary under the C++ facade felt_b200/include/felt_gpu/surface.hpp, which
 * mirrors the Felt reference API (Felt::Surface<D,L>, Felt::Polys<S>). Every entry point below
 * replaces one reference member function; the reference file:line is given beside each one
 * (paths relative to the feltech/Felt source tree). No C++ or torch types cross this boundary:
 * plain pointers, sizes and int status codes (0 = OK, negative = error; fg_last_error() gives
 * the message of the calling thread's last failure). No exceptions cross it.
 *
 * Device memory is owned by the handles; host buffers passed in are owned by the caller.
 * Calls on one handle are issued to that handle's CUDA stream; query calls synchronise it.
 * One host thread per handle at a time.
 *
 * Naming: "layer index" is the reference's TupleIdx layer_idx = layer_id + L, in [0, 2L].
 * Partition indices are row-major (last axis fastest) over the children grid, as in the
 * reference (include/Felt/Impl/Util.hpp:23-40); leaf indices are row-major within a partition.
 */
#ifndef FELT_GPU_H
#define FELT_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FG_API __attribute__((visibility("default")))
#else
#define FG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum {
	FG_OK = 0,
	FG_ERR_ARG = -1,        /* invalid argument or handle                                   */
	FG_ERR_CUDA = -2,       /* CUDA runtime failure (no device, launch failure, ...)        */
	FG_ERR_NOMEM = -3,      /* device or host allocation failed                             */
	FG_ERR_POOL = -4,       /* brick pool exhausted (raise fg_config.brick_capacity)        */
	FG_ERR_NONFINITE = -10, /* a layer id was taken of NaN/inf (reference: iround throws)   */
	FG_ERR_OUTSIDE = -11,   /* a band node would be tracked outside the grid                */
	FG_ERR_INACTIVE = -12,  /* write to an inactive partition (reference: undefined)        */
	FG_ERR_CAPACITY = -13,  /* an output buffer or geometry arena is too small              */
	FG_ERR_TIMEOUT = -14,   /* an update's convergence loop did not settle in 64 iterations,
	                           or a bounded device wait gave up                              */
	FG_ERR_STATE = -15      /* call out of sequence (e.g. update_end without update_start),
	                           or an update of a surface stopped by FG_ERR_TIMEOUT          */
};

/* ---- builtin speed functors ----
 * delta(pos) = [a * curv(pos)] + [n * h(pos, seed)] + [c], each bracket present when its flag
 * is set, summed left to right in FP32. curv is the reference's difference-of-normals mean
 * curvature (include/Felt/Impl/Mixin/NumericMixin.hpp:72-156); h is a fixed 32-bit integer hash
 * of (pos, seed) mapped exactly to [-1, 1). */
enum { FG_SPEED_CONST = 1, FG_SPEED_CURV = 2, FG_SPEED_NOISE = 4 };
typedef struct fg_speed {
	int kind;      /* OR of FG_SPEED_* */
	float c;       /* constant term */
	float a;       /* curvature coefficient */
	float n;       /* noise coefficient */
	uint32_t seed; /* noise seed */
} fg_speed;

typedef struct fg_config {
	size_t brick_capacity; /* bricks (partitions) the device pool can hold; 0 = automatic   */
	size_t vertex_capacity;/* initial polygonisation arena, vertices (simplices: twice that);
	                          0 = 2^20; it grows on demand                                  */
	int launch_mode;       /* how a global update with a builtin speed launches: 0 automatic
	                          (= 1), 1 the whole update as one CUDA graph (its convergence
	                          loop a while node), 2 every kernel launched one by one from
	                          the host, no graphs (per-kernel profilers, debugging)          */
	int dist_split;        /* threads per brick in the first distance pass, in warps per
	                          partition entry (1, 2, 4, 8); 0 = automatic                  */
	int record_passes;     /* threads per brick in the passes that record status changes:
	                          1 a warp, 2 a block per partition entry; 0 = automatic        */
	int autotune;          /* 1: dist_split and record_passes left at 0 take the values
	                          fg_autotune finds for this D, L, partition and device (timed
	                          once per process, or read from the file FELT_TUNE_CACHE names) */
	int delta_kernel;      /* the speed functor of curvature speeds: 1 warps reading the pool,
	                          2 one block per brick staged with its halo in shared memory;
	                          0 = automatic                                                  */
	int fuse_passes;       /* the global update's 2L distance-pass pairs: 1 as 4L launches,
	                          2 as 2L+1 launches (each the second pass of one layer with the
	                          first pass of the next), 3 as two launches: every pass of a
	                          brick in shared memory, the brick staged with a halo of 2L
	                          nodes (where that fits and reaches only the next partitions;
	                          elsewhere as 1); 0 = automatic (= 1)                           */
	int reserved[2];
} fg_config;

typedef struct fg_surface fg_surface;
typedef struct fg_polys fg_polys;
typedef struct fg_batch fg_batch;

FG_API const char* fg_last_error(void);

/* Surface(size, size_partition) (include/Felt/Surface.hpp:163-173). dims in {2,3},
 * layers (L) in {1,2,3,4}; size and part hold `dims` ints. cfg may be NULL. */
FG_API int fg_surface_create(int dims, int layers, const int* size, const int* part,
                      const fg_config* cfg, fg_surface** out);
FG_API int fg_surface_destroy(fg_surface* s);

/* seed(pos) (include/Felt/Surface.hpp:207-241). */
FG_API int fg_seed(fg_surface* s, const int* pos);

/* update(fn) with a builtin speed functor (include/Felt/Surface.hpp:254-296). */
FG_API int fg_update_builtin(fg_surface* s, const fg_speed* speed);

/* update(fn) with a caller-supplied device functor: the facade's templated delta kernel,
 * compiled in the caller's nvcc translation unit, runs between these two calls.
 * fg_update_begin_global performs update_start() and the delta track_children step
 * (include/Felt/Surface.hpp:257-263) and returns the device view the kernel needs;
 * fg_update_finish_global runs update_end_global() (include/Felt/Surface.hpp:739-762). */
typedef struct fg_device_view fg_device_view; /* defined in felt_gpu/device.cuh */
FG_API int fg_update_begin_global(fg_surface* s, const fg_device_view** view, void** stream);
FG_API int fg_update_finish_global(fg_surface* s);

/* update(lo, hi, fn) bounded update with a builtin speed (include/Felt/Surface.hpp:310-386). */
FG_API int fg_update_bounded(fg_surface* s, const int* lo, const int* hi, const fg_speed* speed);

/* update_start() (include/Felt/Surface.hpp:393-399), delta(pos, val) (441-459) and
 * update_end() (404-430): the local update. fg_delta_n applies n deltas in order. */
FG_API int fg_update_start(fg_surface* s);
FG_API int fg_delta(fg_surface* s, const int* pos, float val);
FG_API int fg_delta_n(fg_surface* s, const int* pos, const float* val, size_t n);
FG_API int fg_update_end(fg_surface* s);

/* isogrid().snapshot() (include/Felt/Impl/Mixin/PartitionedMixin.hpp:642-660): dense grid,
 * row-major over the whole isogrid. dst holds n >= prod(size) floats, on the host or, when
 * dst_is_device, in device memory of the surface's GPU. */
FG_API int fg_snapshot(fg_surface* s, float* dst, size_t n, int dst_is_device);

/* Dense snapshot into a host buffer that allocates no memory. No counterpart in the reference:
 * it exists for callers that cannot allocate device memory while they run: processes whose
 * device memory is owned and budgeted by another allocator (a framework's caching allocator or
 * a fixed reservation), and real-time loops that must not enter the driver's allocator, whose
 * cudaMalloc/cudaFree can stall or synchronise the device. It stages through a fixed device
 * array of 2^21 floats (8 MiB) that every GPU loading this library holds until exit; grids with
 * more nodes are rejected with FG_ERR_CAPACITY. Calls share that array (each call writes all
 * it reads), are serialised by a process-wide lock and wait for their copy; calls that
 * overlapped on the GPU would race. The call runs on the surface's device. The first call on a
 * device looks up the array's address on that device and should come before any stream
 * capture. dst holds n >= prod(size) floats. */
FG_API int fg_snapshot_noalloc(fg_surface* s, float* dst, size_t n);

/* isogrid().get(pos) (include/Felt/Impl/Mixin/PartitionedMixin.hpp:594-601). */
FG_API int fg_get(fg_surface* s, const int* pos, float* out);

/* The isogrid's Numeric API from the host, for n positions at once: what the reference's
 * isogrid offers as get(VecDi | VecDf), curv, divergence, grad, gradF, gradB, gradC, gradE
 * (include/Felt/Impl/Mixin/NumericMixin.hpp:72-481; get of a real position is interp) and
 * inside (GridMixin). fg_query takes real positions (n*dims floats), fg_query_nodes nodes
 * (n*dims ints); host arrays. out receives n floats, or n*dims for the gradients (inside: 1 or
 * 0). Results equal a speed functor's calls on the same surface, bit for bit. Positions whose
 * samples leave the grid (undefined in the reference) read the isogrid there as L+1. */
enum {
	FG_Q_GET = 0,
	FG_Q_CURV = 1,
	FG_Q_DIVERGENCE = 2,
	FG_Q_INSIDE = 3,
	FG_Q_GRAD = 4,
	FG_Q_GRADF = 5,
	FG_Q_GRADB = 6,
	FG_Q_GRADC = 7,
	FG_Q_GRADE = 8
};
FG_API int fg_query(fg_surface* s, int what, const float* pos, size_t n, float* out);
FG_API int fg_query_nodes(fg_surface* s, int what, const int* pos, size_t n, float* out);

/* ray(origin, dir) (include/Felt/Surface.hpp:468-616, 1450-1598) for n rays at once: the
 * point where each ray first meets the zero curve, or FLT_MAX in every component (the
 * reference's ray_miss) when it misses. origins, dirs and hits hold n*dims floats each, in host
 * memory; each ray runs on one GPU thread, in the reference's FP32 arithmetic. */
FG_API int fg_ray(fg_surface* s, const float* origins, const float* dirs, size_t n, float* hits);

/* fg_ray with origins, dirs and hits in device memory of the surface's GPU. order_mode chooses
 * how each ray's candidate partitions are put in the reference's order: 0 (the fast default)
 * merges per-axis lists made by a walk kernel, 1 finds each next candidate by a full walk of
 * the planes, 2 merges per-axis cursors. The hits are the same for all three; 1 and 2 exist to
 * test 0. */
FG_API int fg_ray_device(fg_surface* s, const float* origins, const float* dirs, size_t n,
                         float* hits, int order_mode);

/* Surface::save (include/Felt/Surface.hpp:180-183): the surface file in the reference's format
 * (its isogrid through cereal's binary archive: backgrounds, values, leaf and partition lists
 * and lookups, sizes). Writes min(n, cap) bytes to buf (buf may be NULL to ask for the length)
 * and the full length to *n. */
FG_API int fg_save(fg_surface* s, uint8_t* buf, size_t cap, size_t* n);

/* Surface::load (include/Felt/Surface.hpp:185-196): a new surface from a surface file (its
 * dimensions, layers, grid and partition sizes come from the file). The file is checked against
 * the invariants the engine relies on (list entries in range, lookups agreeing with lists,
 * every listed leaf in its own layer, partition lists matching the partitions' leaf lists);
 * a file that breaks one is rejected with FG_ERR_ARG. cfg as for fg_surface_create. */
FG_API int fg_load(const uint8_t* data, size_t n, const fg_config* cfg, fg_surface** out);

/* Geometry of the children (partition) grid: count, size and offset of the children grid. */
FG_API int fg_partitions(fg_surface* s, size_t* count, int* children_size, int* children_offset);

/* isogrid().children().get(p).lookup().list(layer_idx) (LookupMixin.hpp:261-275): the ordered
 * leaf list of one partition. Writes min(n, cap) entries, returns the full count in *n. */
FG_API int fg_layer_list(fg_surface* s, size_t part, int layer_idx, uint32_t* out, size_t cap,
                  size_t* n);

/* isogrid().children().lookup().list(layer_idx) (PartitionedMixin.hpp:104-115): ordered list
 * of partitions tracked in a layer. */
FG_API int fg_partition_list(fg_surface* s, int layer_idx, uint32_t* out, size_t cap, size_t* n);

/* delta(layer_idx) (include/Felt/Surface.hpp:637-640) and status_change(layer_idx) (648-651):
 * partitions touched by the last update. */
FG_API int fg_delta_partitions(fg_surface* s, int layer_idx, uint32_t* out, size_t cap, size_t* n);
FG_API int fg_status_partitions(fg_surface* s, int layer_idx, uint32_t* out, size_t cap, size_t* n);

/* affected() (include/Felt/Surface.hpp:693-696): the affected lookup's partition list for a
 * layer and one partition's ordered leaf list, as left by the last update (calc_affected's
 * rings after a local update). */
FG_API int fg_affected_partitions(fg_surface* s, int layer_idx, uint32_t* out, size_t cap, size_t* n);
FG_API int fg_affected_list(fg_surface* s, size_t part, int layer_idx, uint32_t* out, size_t cap,
                            size_t* n);

/* children().get(p).is_active() and background() (GridMixin.hpp:56-69). */
FG_API int fg_partition_state(fg_surface* s, size_t part, int* active, float* background);

/* stats() (include/Felt/Surface.hpp:623-629). */
FG_API int fg_stats(fg_surface* s, size_t* active_isogrid_partitions, size_t* active_delta_partitions);

/* Iterations of the convergence loop (distance passes, flush, expansion) the last global or
 * local update ran, the first one included (the reference's loop at Surface.hpp:747-761 and
 * 417-428 does not count them). */
FG_API int fg_update_iterations(fg_surface* s, int* iterations);

/* Narrow-band node count at the start of the last update: sum over the 2L+1 layers. */
FG_API int fg_band_size(fg_surface* s, size_t* n);

/* Canonical state encoding used by parity tests (uint32 words):
 *   D, L, P (partition count);
 *   per partition: active, background (float bits), then per layer: n, n leaf indices;
 *   per layer: isogrid partition list (n, entries);
 *   per layer: delta partition list; per layer: status-change partition list.
 * Writes min(total, cap) words and the full word count in *n. */
FG_API int fg_dump(fg_surface* s, uint32_t* out, size_t cap, size_t* n);

/* ---- Polys<Surface> (include/Felt/Polys.hpp) ---- */
FG_API int fg_polys_create(fg_surface* s, fg_polys** out);   /* Polys.hpp:58-84   */
FG_API int fg_polys_destroy(fg_polys* p);
FG_API int fg_polys_notify(fg_polys* p);                       /* Polys.hpp:92-133  */
FG_API int fg_polys_march(fg_polys* p);                        /* Polys.hpp:138-165 */
FG_API int fg_polys_invalidate(fg_polys* p);                   /* Polys.hpp:171-191 */
/* Poly::Single::march of one partition's child (Poly.hpp:138-147), activating or resetting it
 * first as Polys::march does (Polys.hpp:149-154). */
FG_API int fg_polys_march_partition(fg_polys* p, size_t part);
FG_API int fg_polys_changes(fg_polys* p, uint32_t* out, size_t cap, size_t* n); /* Polys.hpp:198-201 */
/* children().get(part).{vtxs(),spxs(),is_active()} (Poly.hpp:155-186). vtx receives per vertex
 * D position floats then, in 3D, D normal floats; spx receives D uint32 indices per simplex. */
FG_API int fg_polys_partition(fg_polys* p, size_t part, float* vtx, size_t vtx_cap, uint32_t* spx,
                       size_t spx_cap, size_t* nv, size_t* ns, int* active);
/* The geometry of several partitions in one call (what a viewer reads after a march, e.g. the
 * partitions of fg_polys_changes): vertices and simplices of parts[0..n) concatenated in that
 * order, counts[2*i] / counts[2*i+1] the vertex / simplex count of parts[i]. Simplex indices
 * stay local to their partition, as in children().get(p).spxs(). With vtx and spx NULL only the
 * counts and totals are returned. */
FG_API int fg_polys_gather(fg_polys* p, const uint32_t* parts, size_t n, float* vtx,
                           size_t vtx_cap, uint32_t* spx, size_t spx_cap, uint32_t* counts,
                           size_t* nv, size_t* ns);

/* Totals over all partitions. */
FG_API int fg_polys_totals(fg_polys* p, size_t* vertices, size_t* simplices);

/* ---- batches: many independent surfaces advanced by the same kernel launches ----
 * The reference runs one Surface at a time; a batch holds n surfaces that share D, L and the
 * partition shape but may differ in grid size, and every update / polygonisation call advances
 * all of them in the same launches. Per surface the results are exactly those of a separate
 * fg_surface (same lists, orders and values). sizes holds n*dims ints. */
FG_API int fg_batch_create(int dims, int layers, const int* part, size_t n, const int* sizes,
                           const fg_config* cfg, fg_batch** out);
FG_API int fg_batch_destroy(fg_batch* b);
/* seed(pos) of every surface (centres: n*dims ints), one seed per surface. */
FG_API int fg_batch_seed(fg_batch* b, const int* centres);
/* update(fn) of every surface with its own builtin speed (speeds: n entries). */
FG_API int fg_batch_update(fg_batch* b, const fg_speed* speeds);
/* Polys over the batch: notify / march / invalidate for all surfaces at once. */
FG_API int fg_batch_polys_notify(fg_batch* b);
FG_API int fg_batch_polys_march(fg_batch* b);
FG_API int fg_batch_polys_invalidate(fg_batch* b);
/* Per-surface queries, as the fg_surface ones. */
FG_API int fg_batch_snapshot(fg_batch* b, size_t surface, float* dst, size_t n);
FG_API int fg_batch_dump(fg_batch* b, size_t surface, uint32_t* out, size_t cap, size_t* n);
/* Surface::save (include/Felt/Surface.hpp:180-183) of one surface of a batch: the same file as
 * fg_save writes (min(n, cap) bytes into buf, which may be NULL; the full length in *n). */
FG_API int fg_batch_save(fg_batch* b, size_t surface, uint8_t* buf, size_t cap, size_t* n);
/* Surface::load (include/Felt/Surface.hpp:185-196) into one surface of a batch, which must be
 * empty (never seeded, or with no active partition and every list empty; else FG_ERR_STATE) and
 * have the file's grid and partition size: a checkpoint taken with fg_batch_save or fg_save
 * comes back into any batch, e.g. a served surface set aside and later resumed. Its bricks come
 * from the batch's pool (FG_ERR_POOL when too few are free). The batch's polygonisation sees the
 * restored partitions after fg_batch_polys_invalidate, as a Polys built for a loaded surface
 * does after Polys::invalidate (include/Felt/Polys.hpp:171-180). */
FG_API int fg_batch_restore(fg_batch* b, size_t surface, const uint8_t* data, size_t n);
/* fg_query / fg_query_nodes on one surface of a batch. */
FG_API int fg_batch_query(fg_batch* b, size_t surface, int what, const float* pos, size_t n,
                          float* out);
FG_API int fg_batch_query_nodes(fg_batch* b, size_t surface, int what, const int* pos, size_t n,
                                float* out);
FG_API int fg_batch_ray(fg_batch* b, size_t surface, const float* origins, const float* dirs,
                         size_t n, float* hits);
FG_API int fg_batch_polys_partition(fg_batch* b, size_t surface, size_t part, float* vtx,
                                    size_t vtx_cap, uint32_t* spx, size_t spx_cap, size_t* nv,
                                    size_t* ns, int* active);
FG_API int fg_batch_polys_changes(fg_batch* b, size_t surface, uint32_t* out, size_t cap,
                                  size_t* n);
FG_API int fg_batch_polys_totals(fg_batch* b, size_t* vertices, size_t* simplices);
FG_API int fg_batch_node_updates(fg_batch* b, unsigned long long* n);
/* Whether a surface has been stopped. The reference's convergence loop (Surface.hpp:752-760)
 * has no bound and, where the band meets the grid edge, its layer changes can oscillate
 * forever; after 64 iterations the surfaces still changing are stopped (left as they are, never
 * worked on again) so the rest of the batch completes. A single fg_surface reports the same
 * event as FG_ERR_TIMEOUT from the update, and FG_ERR_STATE from later updates. */
FG_API int fg_batch_surface_stopped(fg_batch* b, size_t surface, int* stopped);
/* Pauses (paused != 0) or resumes one surface of a batch. No counterpart in the reference: a
 * server retires a finished request this way, so later batch updates, notifies and marches skip
 * it and its state stays exactly as after its own last update (equal to a separate fg_surface
 * advanced by the same updates). */
FG_API int fg_batch_pause(fg_batch* b, size_t surface, int paused);
FG_API int fg_batch_work_units(fg_batch* b, unsigned long long* out, size_t n);
FG_API int fg_batch_stream(fg_batch* b, void** stream);

/* ---- serving: continuous batching of level-set requests ----
 * No counterpart in the reference, which advances one Surface at a time. A server owns one
 * long-lived pool of `slots` surfaces, each sized for grids up to max_size, sharing one brick
 * pool, and a worker thread that advances every surface in flight by one batched
 * Surface::update (include/Felt/Surface.hpp:254-296) per step, with Polys::notify
 * (include/Felt/Polys.hpp:92-133) for requests that want polygons and Polys::march
 * (Polys.hpp:138-165) when one of them has had its last update. Requests that arrive while
 * others run take freed slots at the next step boundary (reset to the request's grid, seeded,
 * then advanced in the same launches as the rest), so their work overlaps on the device. Each
 * request's result equals a separate fg_surface given the same seed and updates.
 * Admission: a request reserves the bricks its band can reach (the partitions within
 * L + 2 + steps * max(1, largest |delta| of its speed) cells of its seed, clipped to its grid;
 * fg_request_bricks) and is rejected at submission (FG_ERR_CAPACITY) when the reservations of
 * requests queued and in flight would exceed the brick pool. */
typedef struct fg_server fg_server;
typedef struct fg_server_config {
	int dims;               /* 2 or 3 */
	int layers;             /* L, 1..4 */
	int part[3];            /* partition size */
	int max_size[3];        /* largest grid a request may ask for (each slot's capacity) */
	size_t slots;           /* surfaces in flight at most */
	size_t brick_capacity;  /* bricks in the shared pool; 0 = budget_bytes / bytes per brick */
	double budget_bytes;    /* device bytes of the brick pool, when brick_capacity is 0 */
	size_t vertex_capacity; /* initial polygon arena (vertices), 0 = 2^20; grows on demand */
	int keep_outputs;       /* keep each result's state dump and polygons until released */
	int reserved[7];
} fg_server_config;
typedef struct fg_request {
	int size[3];            /* grid size */
	int centre[3];          /* seed position (Surface::seed, Surface.hpp:207-241) */
	fg_speed speed;         /* builtin speed of every update */
	int steps;              /* global updates, >= 1 */
	int polygonise;         /* march the polygons after the last update */
	uint64_t tag;           /* the caller's id, returned with the result */
} fg_request;
typedef struct fg_result {
	uint64_t tag;
	int status;             /* FG_OK; FG_ERR_TIMEOUT when the surface was stopped (its update's
	                           convergence loop did not settle); another code on a fault */
	int steps_done;
	double t_submit, t_admit, t_done;   /* seconds on the server's clock (fg_server_now) */
	unsigned long long node_updates;    /* band size at the start of each of its updates */
	unsigned long long vertices, simplices;  /* its polygons, when it asked for them */
} fg_result;
typedef struct fg_server_stats {
	unsigned long long submitted, admitted, rejected;  /* at submission */
	unsigned long long started;          /* taken into a slot */
	unsigned long long completed;        /* finished (stopped surfaces included) */
	unsigned long long failed;           /* ended by a fault */
	unsigned long long steps;            /* batched steps run */
	unsigned long long node_updates;     /* of finished requests */
	unsigned long long capacity_bricks, reserved_bricks, peak_reserved_bricks, peak_used_bricks;
	unsigned long long queued, in_flight;
	int fault_code;
	int reserved[7];
} fg_server_stats;
FG_API int fg_server_create(const fg_server_config* cfg, fg_server** out);
/* Stops the worker after its current step and frees the pool. */
FG_API int fg_server_destroy(fg_server* s);
/* Seconds since the server was created (the clock of fg_result's times). */
FG_API int fg_server_now(fg_server* s, double* t);
/* Queues a request, or rejects it with FG_ERR_CAPACITY (budget reserved, or a grid larger
 * than max_size). Any thread. */
FG_API int fg_server_submit(fg_server* s, const fg_request* r);
/* Up to cap finished results, oldest first (waits up to wait_s seconds for the first). */
FG_API int fg_server_poll(fg_server* s, fg_result* out, size_t cap, size_t* n, double wait_s);
FG_API int fg_server_get_stats(fg_server* s, fg_server_stats* out);
/* With keep_outputs: a finished request's state (the fg_dump encoding) and its polygons (every
 * partition's vertices and simplices concatenated in partition order, counts[2p], counts[2p+1]
 * the vertex and simplex count of partition p); fg_server_release drops them. */
FG_API int fg_server_result_dump(fg_server* s, uint64_t tag, uint32_t* out, size_t cap, size_t* n);
FG_API int fg_server_result_polys(fg_server* s, uint64_t tag, float* vtx, size_t vtx_cap,
                                  uint32_t* spx, size_t spx_cap, uint32_t* counts,
                                  size_t counts_cap, size_t* nv, size_t* ns, size_t* nparts);
FG_API int fg_server_release(fg_server* s, uint64_t tag);
/* The bricks a request reserves on a server of this configuration (host arithmetic only), and
 * the device bytes of one brick of the pool. */
FG_API int fg_request_bricks(const fg_server_config* cfg, const fg_request* r,
                             unsigned long long* bricks);
FG_API int fg_brick_bytes(int dims, int layers, const int* part, double* bytes);

/* Launch tuning by measurement (no counterpart in the reference). fg_autotune_candidates lists
 * the (dist_split, record_passes) pairs worth timing for a partition shape (pairs[2i],
 * pairs[2i+1]). fg_autotune times each on a scratch surface of this dimension, layer count and
 * partition shape on the current device (a sphere grown to a quarter of a grid of 64..256 per
 * axis, then curvature-plus-constant updates) and writes the fastest pair into cfg's
 * dist_split and record_passes (other fields untouched); ms receives each candidate's device
 * time per update in candidate order and *n their number, 0 when the result came from the
 * process's cache or the FELT_TUNE_CACHE file (force = 1 times again). The knobs change launch
 * shapes only: results are the same under every pair. */
FG_API int fg_autotune_candidates(int dims, const int* part, int* pairs, size_t cap, size_t* n);
FG_API int fg_autotune(int dims, int layers, const int* part, int force, fg_config* cfg,
                       double* ms, size_t ms_cap, size_t* n);
/* The launch tuning in effect on a surface or batch (5 values): out[0] launch mode (1 one graph,
 * 2 phase by phase), out[1] dist_split, out[2] record_passes, out[3] delta kernel (1 direct,
 * 2 staged), out[4] distance passes (1 separate, 2 fused). */
FG_API int fg_surface_tuning(fg_surface* s, int* out);
FG_API int fg_batch_tuning(fg_batch* b, int* out);

/* ---- instrumentation (no counterpart in the reference; Surface.hpp has no timers) ----
 * fg_node_updates: narrow-band node-updates processed by all global updates of a surface so
 * far (band size at the start of each update, summed). fg_launch_count: kernels this library
 * has launched in the process. fg_profile_*: per-kernel device time from CUDA events recorded
 * around every launch while profiling is enabled. */
FG_API int fg_node_updates(fg_surface* s, unsigned long long* n);
/* Work units processed so far on the surface's pool: [0] band nodes through the distance
 * passes, [1] zero-layer nodes through the speed functor, [2] leaf edits of the status-change
 * flush, [3] cells marched by Polys. Writes min(n, 8) counters. */
FG_API int fg_work_units(fg_surface* s, unsigned long long* out, size_t n);
/* The CUDA stream (cudaStream_t) every call on this surface is issued to. */
FG_API int fg_surface_stream(fg_surface* s, void** stream);
/* Dimensions, layers, grid size and partition size of a surface (size and part: dims ints each,
 * either may be NULL): what a surface made by fg_load was given by its file. */
FG_API int fg_surface_info(fg_surface* s, int* dims, int* layers, int* size, int* part);
FG_API int fg_launch_count(long long* n);
FG_API int fg_profile_enable(int on);
FG_API int fg_profile_reset(void);
/* Limits the event bracketing to launches of one kernel (NULL or "" = every kernel), so that a
 * kernel can be timed without events around every other launch. */
FG_API int fg_profile_only(const char* kernel);
FG_API int fg_profile_count(size_t* n);
FG_API int fg_profile_entry(size_t i, char* name, size_t name_cap, double* ms, long long* launches);

#ifdef __cplusplus
}
#endif
#endif
