/*
 * enterprise_b200 — C ABI of the B200-native (sm_100a) breadth-first search.
 *
 * This is the drop-in boundary for Enterprise's GPU BFS. The reference
 * exposes one host entry point,
 *     template<vertex_t,index_t> int bfs_gpu_coalescing_mem(
 *         vertex_t* src_list, index_t* beg_pos, vertex_t* csr,
 *         index_t vert_count, index_t edge_count, index_t gpu_id)
 * (bfs_gpu_opt.cuh:293-300), fed by the CSR loader graph<...>::graph
 * (graph.hpp:33-118) and called from main.cu:80-86. That function uploads
 * the CSR (allocator.cuh:35-150), runs 64 BFS traversals and only prints.
 * Here the same work is split into explicit steps a foreign-function layer
 * can bind: load / create a device graph, run one or many traversals,
 * read depths (and optionally parents) back, destroy.
 *
 * Conventions
 *  - Every function returns an int status (ENT_OK == 0). Nothing calls
 *    exit(); the reference's H_ERR (comm.h:34-45) aborted the process.
 *    ent_last_error() returns a thread-local message for the last failure.
 *  - Host arrays passed in are borrowed (read-only, never freed).
 *  - Depths are int32; unreached vertices hold -1 (all ones, mirroring the
 *    reference's INFTY = 0xFF for its uint8 depth_t, comm.h:69, comm.h:131).
 *  - Parents are int32; parent[src] == src; unreached vertices hold -1.
 *  - A graph handle owns its device memory. Calls on one handle are
 *    serialised internally; distinct handles may be used from different
 *    host threads.
 *  - Vertex ids are int32 (V < 2^31). Offsets are int64 (E may exceed 2^31).
 */
#ifndef ENTERPRISE_B200_H
#define ENTERPRISE_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ENT_ABI_VERSION 5

enum ent_status {
  ENT_OK = 0,
  ENT_ERR_INVALID_ARG = 1,
  ENT_ERR_CUDA = 2,
  ENT_ERR_OOM = 3,
  ENT_ERR_IO = 4,
  ENT_ERR_FORMAT = 5,
  ENT_ERR_TIMEOUT = 6,
  ENT_ERR_INTERNAL = 7,
  ENT_ERR_UNSUPPORTED = 8,
  ENT_ERR_ADMISSION = 9
};

/* Direction policy (reference rule: inspector.cuh:486-521). */
enum ent_policy {
  ENT_POLICY_BEAMER = 0,    /* alpha/beta direction switching, both ways  */
  ENT_POLICY_REFERENCE = 1, /* TD->BU once when frontier edges >= ratio*E */
  ENT_POLICY_TD_ONLY = 2,   /* top-down every level                       */
  ENT_POLICY_BU_ONLY = 3    /* bottom-up every level                      */
};

/* How the level loop is driven. */
enum ent_loop {
  ENT_LOOP_GRAPH = 0, /* whole traversal = one CUDA graph launch with a
                         device-side while node (no host round trip)   */
  ENT_LOOP_HOST = 1   /* host launches each level and polls a flag     */
};

typedef struct ent_bfs_opts {
  int32_t policy;        /* enum ent_policy                                */
  int32_t loop;          /* enum ent_loop                                  */
  double alpha;          /* Beamer: TD->BU when m_f > m_u / alpha          */
  double beta;           /* Beamer: BU->TD when n_f < V / beta (shrinking) */
  double ref_ratio;      /* reference rule ratio (0.3, inspector.cuh:497)  */
  int32_t small_max;     /* degree <  small_max -> thread tier (ref 32)    */
  int32_t large_min;     /* degree >  large_min -> CTA tier (ref 1024)     */
  int32_t hub_slots;     /* shared-memory hub cache slots, power of two,
                            0 disables (ref 1536/1920, comm.h:176-177)     */
  int32_t chunk_edges;   /* edges per CTA chunk of a large TD vertex       */
  int32_t blocks_per_sm; /* resident CTAs per SM for the level kernels,
                            0 = occupancy maximum                          */
  /* batched (bitwise multi-source) traversal */
  double batch_alpha;      /* bottom-up when frontier edges*alpha > unfinished edges */
  int32_t batch_small_max; /* bottom-up: degree < this -> lane group per vertex     */
  int32_t batch_large_min; /* bottom-up: degree >= this -> CTA per vertex           */
  int32_t batch_heavy;     /* top-down: degree >= this -> all CTAs share the vertex */
  /* small-frontier ("narrow") mode of the single-source traversal: while the
     top-down frontier stays small, one thread-block cluster runs level after
     level inside a single launch. Entered when the frontier has at most
     narrow_max_frontier vertices, narrow_max_edges edges and no vertex of
     degree > narrow_max_degree; left when it grows past twice the first two
     or meets such a vertex. narrow_max_frontier = 0 disables the mode. */
  int32_t narrow_max_frontier;
  int32_t narrow_max_edges;
  int32_t narrow_max_degree;
  int32_t narrow_cluster;  /* CTAs in the cluster (1..16), 0 = largest that fits */
  int32_t fault_inject;    /* test hook, 0 in use. 1: the first tile of each frontier
                              classification never publishes its prefix, so the
                              tiles that wait for it run out their bounded spin
                              (about a second) and the traversal returns
                              ENT_ERR_TIMEOUT with the context still usable */
  /* Batches on deep graphs (grids, road-like graphs): their thousands of small
     levels would cost a grid-wide bitwise batch two launches each, and sources
     on such graphs share little frontier, so the batch runs instead as
     concurrent single-source traversals ("lanes"), each running its small
     frontiers inside its own thread-block cluster of batch_deep_cluster CTAs,
     as many lanes as the GPU holds clusters (or batch_deep_lanes), each
     writing its source's row. batch_deep: 0 = never, 1 = auto (when a probe
     traversal of the graph, run once per graph by its first batch, has at
     least batch_deep_levels levels), 2 = always. */
  int32_t batch_deep;
  int32_t batch_deep_levels;
  int32_t batch_deep_cluster; /* CTAs per lane's cluster (1..16); 0 = per batch, the
                                 largest power of two in [4, 16] whose n_src clusters
                                 fit the SMs                                           */
  int32_t batch_deep_lanes;   /* concurrent lanes at most, 0 = as many as fit          */
} ent_bfs_opts;

typedef struct ent_stats {
  int64_t reached_vertices; /* reference report(): agg_tr_v (validate.h:106-127) */
  int64_t traversed_edges;  /* reference report(): agg_tr_edges = sum of degrees of
                               reached vertices (directed CSR entries)           */
  int32_t levels;           /* number of non-empty levels = max depth + 1         */
  int32_t td_levels;        /* levels expanded top-down                           */
  int32_t bu_levels;        /* levels expanded bottom-up                          */
  int32_t status;           /* device status word (0 ok)                          */
  double device_ms;         /* CUDA-event time of the traversal on the device     */
  int32_t narrow_levels;    /* of td_levels, those run inside the small-frontier
                               cluster kernel                                     */
  int32_t launches;         /* kernels launched by this traversal                 */
} ent_stats;

typedef struct ent_graph ent_graph; /* device-resident CSR + traversal state */
typedef struct ent_csr ent_csr;     /* host-resident CSR owned by the library */

/* ---------------------------------------------------------------- misc --- */
const char* ent_last_error(void);
int ent_abi_version(void);
void ent_bfs_opts_default(ent_bfs_opts* opts);
/* Number of kernels this library has launched in this process (all devices). */
int64_t ent_kernel_launch_count(void);

/* ------------------------------------------------------- host CSR ------- */
/* Replaces graph<long,long,double,int,int,double>(beg,csr,NULL)
 * (graph.hpp:33-118): reads <X>_beg_pos.bin (int64[V+1]) and <X>_csr.bin.
 * The csr file may hold int64 (the reference's format, graph.hpp:46-47) or
 * int32 entries; the width is detected from file size vs beg_pos[V].
 * Offsets are validated (monotone, beg_pos[0]==0) and ids checked < V. */
int ent_csr_load(const char* beg_pos_path, const char* csr_path, ent_csr** out);
/* Writes the reference's int64 format (both files int64). */
int ent_csr_save(const ent_csr* g, const char* beg_pos_path, const char* csr_path);
/* Builds a CSR from caller arrays (copied). */
int ent_csr_from_arrays(const int64_t* beg_pos, const int32_t* csr, int64_t vert_count,
                        int64_t edge_count, ent_csr** out);
/* Builds a canonical undirected CSR from an edge list: both directions added,
 * self loops and duplicates removed, rows sorted ascending. */
int ent_csr_from_edges(const int64_t* src, const int64_t* dst, int64_t n_edges,
                       int64_t vert_count, ent_csr** out);
int64_t ent_csr_vert_count(const ent_csr* g);
int64_t ent_csr_edge_count(const ent_csr* g);
const int64_t* ent_csr_beg_pos(const ent_csr* g);
const int32_t* ent_csr_adj(const ent_csr* g);
void ent_csr_free(ent_csr* g);

/* Seeded generators on the host (OpenMP). Output: canonical undirected CSR
 * with vertex ids scrambled by a seeded bijection. */
int ent_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                 uint64_t seed, ent_csr** out);
int ent_gen_grid(int64_t width, int64_t height, double drop_prob, uint64_t seed,
                 ent_csr** out);
int ent_gen_er(int64_t vert_count, double mean_degree, uint64_t seed, ent_csr** out);
/* Seeded distinct non-isolated sources (count <= number of such vertices). */
int ent_pick_sources(const int64_t* beg_pos, int64_t vert_count, uint64_t seed,
                     int32_t count, int32_t* out);
/* The reference's source rule (main.cu:55-78): glibc rand()%V from the
 * process's current rand() state, distinct, non-isolated. */
int ent_pick_sources_compat(const int64_t* beg_pos, int64_t vert_count, int32_t count,
                            int32_t* out);

/* ------------------------------------------------------- device graph --- */
/* Uploads a CSR to GPU `gpu_id` and allocates traversal state
 * (replaces allocator<>::alloc_array, allocator.cuh:35-150). */
int ent_graph_create(const int64_t* beg_pos, const int32_t* csr, int64_t vert_count,
                     int64_t edge_count, int32_t gpu_id, ent_graph** out);
int ent_graph_from_csr(const ent_csr* g, int32_t gpu_id, ent_graph** out);
/* Loads <beg_pos.bin> (int64[V+1]) and <csr.bin> (int64[E] or int32[E]) into
 * a device graph without a host copy of the CSR: chunks of csr.bin are read
 * by several threads into pinned buffers, copied asynchronously and narrowed
 * to int32 on the GPU while the next chunk is read (replaces the reference's
 * graph loader with its serial narrowing loop, graph.hpp:33-118, and its
 * upload, allocator.cuh:107-120). Format rules and errors as ent_csr_load. */
int ent_graph_load(const char* beg_pos_path, const char* csr_path, int32_t gpu_id, ent_graph** out);
/* Generates a graph directly on the GPU (same edges as the host generators,
 * bit-identical CSR). */
int ent_graph_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                       uint64_t seed, int32_t gpu_id, ent_graph** out);
int ent_graph_gen_grid(int64_t width, int64_t height, double drop_prob, uint64_t seed,
                       int32_t gpu_id, ent_graph** out);
int ent_graph_gen_er(int64_t vert_count, double mean_degree, uint64_t seed,
                     int32_t gpu_id, ent_graph** out);
/* Builds the canonical undirected CSR of a caller's edge list on the GPU:
 * both directions, self loops and duplicates dropped, rows ascending (the
 * same CSR as ent_csr_from_edges; the reference builds CSR offline with its
 * text converter, tuple_text_to_binary_csr/). src/dst: HOST arrays of n_edges
 * ids in [0, vert_count); an endpoint outside returns ENT_ERR_FORMAT naming
 * the first such edge. */
int ent_graph_from_edges(const int64_t* src, const int64_t* dst, int64_t n_edges, int64_t vert_count,
                         int32_t gpu_id, ent_graph** out);
int64_t ent_graph_vert_count(const ent_graph* g);
int64_t ent_graph_edge_count(const ent_graph* g);
int32_t ent_graph_device(const ent_graph* g);  /* the graph's GPU */
/* Device bytes held by the graph's resident arrays (offsets, the two column
 * arrays, degrees, the active bitmap and the lead entries; traversal
 * workspaces come on top). The reference prints its allocation total as
 * "GPU alloc space: N bytes" (allocator.cuh:149). */
int64_t ent_graph_device_bytes(const ent_graph* g);
/* Device buffers for callers without a CUDA runtime of their own (a
 * foreign-function binding, the command line): bytes on GPU gpu, for the
 * *_device calls and ent_validate. Free with ent_device_free. */
int ent_device_alloc(int32_t gpu, size_t bytes, void** out);
int ent_device_free(void* ptr);
/* Copies the device CSR to caller host arrays (V+1 and E entries). */
int ent_graph_download(const ent_graph* g, int64_t* beg_pos, int32_t* csr);
/* Device pointers of the resident CSR (for callers that keep work on GPU). */
int ent_graph_device_csr(const ent_graph* g, const int64_t** beg_pos_dev,
                         const int32_t** csr_dev);
int ent_graph_set_opts(ent_graph* g, const ent_bfs_opts* opts);
int ent_graph_get_opts(const ent_graph* g, ent_bfs_opts* opts);
int ent_graph_destroy(ent_graph* g);

/* ------------------------------------------------------- traversal ------ */
/* One direction-optimising BFS from `src`. depth_out / parent_out are HOST
 * arrays of V int32 (either may be NULL). stats may be NULL. */
int ent_bfs(ent_graph* g, int32_t src, int32_t* depth_out, int32_t* parent_out,
            ent_stats* stats);
/* Same traversal; results stay on the device. depth_dev / parent_dev are
 * device arrays of V int32 on the graph's GPU (parent_dev may be NULL).
 * The call is asynchronous on `stream` (a cudaStream_t, NULL = the graph's
 * own stream) unless stats is non-NULL, which synchronises. */
int ent_bfs_device(ent_graph* g, int32_t src, int32_t* depth_dev, int32_t* parent_dev,
                   void* stream, ent_stats* stats);
/* One traversal per source, in order, with each source's depths copied to a
 * HOST array: the reference's per-source loop (bfs_gpu_opt.cuh:370-431:
 * reset, traverse, depth D2H) as one call. depth_out[i] (V int32) receives
 * source i's depths; an entry may be NULL (no copy) or repeat an earlier one
 * (the later source's depths win). The copy of source i overlaps the
 * traversal of source i+1, which needs page-locked host arrays to overlap
 * (pageable ones still work, serialised). stats (n_src entries) may be NULL.
 * Returns once every copy has landed. */
int ent_bfs_many(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* const* depth_out,
                 ent_stats* stats);
/* The same loop with the reference's own depth type: depth_out[i] is a HOST
 * array of V bytes (depth_t = unsigned char, comm.h:69), depth d as d and
 * unreached as 255 (INFTY, comm.h:131), a quarter of the bytes to copy. The
 * reference wraps depths above 254 around; here a source whose traversal
 * goes deeper returns ENT_ERR_UNSUPPORTED (its row then holds the low byte
 * of each depth; the other sources' rows are complete). */
int ent_bfs_many_u8(ent_graph* g, const int32_t* src, int32_t n_src, uint8_t* const* depth_out,
                    ent_stats* stats);

/* Per-level trace of one traversal (tracing / profiling aid). Runs the level
 * loop host-driven with CUDA events around each kernel; depths are the same
 * as ent_bfs. out holds max_levels entries; *n_levels gets the count. */
typedef struct ent_level_trace {
  int32_t level;             /* depth of the frontier expanded                */
  int32_t direction;         /* 0 top-down, 1 bottom-up                       */
  int32_t bu_sweep;          /* bottom-up over every vertex (first BU level)  */
  int32_t pad;
  int64_t frontier_vertices; /* n_f of the frontier expanded                  */
  int64_t frontier_edges;    /* m_f                                           */
  int64_t unvisited_queued;  /* BU: unvisited vertices in the tier queues     */
  double expand_ms;
  double inspect_ms;
} ent_level_trace;
int ent_bfs_trace(ent_graph* g, int32_t src, ent_level_trace* out, int32_t max_levels, int32_t* n_levels,
                  ent_stats* stats);

/* BFS that allocates nothing. No counterpart in the reference: it exists for
 * callers that may not allocate GPU memory when they traverse — code on a
 * latency-critical path, where cudaMalloc/cudaFree can synchronise the device
 * and stall other streams, and plug-ins in processes whose GPU memory is
 * owned by another allocator or a fixed budget. The caller passes the CSR
 * (beg_pos: V+1 int64, csr: int32, valid ids, e.g. from ent_graph_device_csr)
 * and depth_dev (V int32) in device memory of the current device; the
 * traversal's scratch is a static array inside this library on every GPU that
 * loads it (about 8.5 MB) and limits V to ENT_NOALLOC_MAX_VERTICES; larger
 * graphs return ENT_ERR_INVALID_ARG. The first call on a device looks up the
 * array's device address, so make that first call before any stream capture.
 * That first call may also be when CUDA loads this library's GPU code onto the
 * device (modules load lazily by default), which places the array there and
 * so takes its 8.5 MB of device memory, and fails if that memory is not free:
 * make one call while the process initialises, before it enters the code that
 * may not allocate. The address is valid only in the CUDA context it was
 * looked up in; a caller that also calls from a context of its own (a
 * driver-API plug-in) gets one more lookup, once, in that context.
 * All calls share the array: calls whose work overlaps on one GPU race and
 * give wrong results, so serialise them. Synchronous on `stream` (NULL = the
 * default stream). */
#define ENT_NOALLOC_MAX_VERTICES (1 << 20)
int ent_bfs_noalloc(const int64_t* beg_pos_dev, const int32_t* csr_dev, int64_t vert_count,
                    int32_t src, int32_t* depth_dev, void* stream);

/* Graph500-style validation of one traversal's result on the GPU, every
 * vertex and edge (the reference's validate() spot-checks one random vertex,
 * validate.h:34-103). depth_dev / parent_dev: device arrays of V int32 on the
 * graph's GPU (parent_dev may be NULL). Depth rules, in order: -1 depth[src]
 * != 0; per vertex v ascending: -2 depth < -1, -3 depth 0 but v != src, at the
 * first edge of v's row that breaks one: -4 exactly one end reached, -5 both
 * reached but depths differ by more than 1; -6 v reached at depth > 0 with no
 * neighbour one level up. Parent rules: -1 parent[src] != src or depth[src]
 * != 0; per v != src ascending: -2 unreached v with a parent, -3 parent out
 * of range, -4 depth[parent] != depth[v] - 1, -5 (parent, v) not an edge.
 * *_code = 0 when all hold, else the rule broken at the smallest offending
 * vertex *_bad (-1 when none). Synchronous. */
int ent_validate(ent_graph* g, int32_t src, const int32_t* depth_dev, const int32_t* parent_dev,
                 int32_t* depth_code, int64_t* depth_bad, int32_t* parent_code, int64_t* parent_bad);

/* Many sources at once with bitwise frontiers (one bit per source per vertex
 * in a shared status word). depth_out: HOST array n_src x V int32, source-major
 * (row s is the depth array of src[s]); may be NULL. stats: n_src entries or
 * NULL. Depths are identical to n_src calls of ent_bfs. */
int ent_bfs_batch(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_out,
                  ent_stats* stats);
/* Batched traversal with device-resident output (n_src x V int32 on the GPU). */
int ent_bfs_batch_device(ent_graph* g, const int32_t* src, int32_t n_src,
                         int32_t* depth_dev, void* stream, ent_stats* stats);
/* The same two calls with the reference's own depth type: rows of n_src x V
 * bytes (depth_t = unsigned char, comm.h:69; 255 = unreached, comm.h:131), a
 * quarter of the bytes to write and to copy. A source whose traversal goes
 * deeper than 254 levels makes the call return ENT_ERR_UNSUPPORTED (its row
 * holds the low byte of each depth; the other rows are complete), where the
 * reference wraps around. */
int ent_bfs_batch_u8(ent_graph* g, const int32_t* src, int32_t n_src, uint8_t* depth_out,
                     ent_stats* stats);
int ent_bfs_batch_device_u8(ent_graph* g, const int32_t* src, int32_t n_src,
                            uint8_t* depth_dev, void* stream, ent_stats* stats);

/* Host-driven batched run with CUDA events per level (tracing aid). Entry
 * n-1 with level == -1 times the final depth flush. */
int ent_bfs_batch_trace(ent_graph* g, const int32_t* src, int32_t n_src, int32_t* depth_dev,
                        ent_level_trace* out, int32_t max_levels, int32_t* n_levels);

/* Many graphs of uneven sizes in one launch: graphs[k] gets n_src[k] sources
 * from src (concatenated). depth_out[k] is a HOST array n_src[k] x V_k or
 * NULL. All graphs must live on the same GPU; a graph may be listed more than
 * once (several source sets). */
int ent_bfs_multi(ent_graph* const* graphs, int32_t n_graphs, const int32_t* src,
                  const int32_t* n_src, int32_t* const* depth_out);

/* The same as a reusable plan: create once, run many times (one graph
 * launch; device_ms may be NULL), read each graph's n_src[k] x V_k depths,
 * destroy. The graphs are grouped by the width class of their request (64-bit
 * words per vertex: ceil(n_src / 64) rounded up to a power of two), and each
 * class runs as ONE batched traversal over the disjoint union of its graphs:
 * create copies the graphs' CSR into one union per class (vertex and edge
 * offsets per graph, the plan's descriptor table) and seeds source slot s at
 * the s-th source of every graph of the class; a graph with fewer sources
 * than the class's widest request repeats its own (slot s at source
 * s % n_src[k]). Every level then runs one expand and one commit for all
 * graphs of a class over the whole GPU. Create also measures each union's
 * direction threshold (batch alpha: the member with the most edges' own value
 * and 2, 4, 8, 16, 32, two host-driven runs each, the fastest kept; unions
 * deeper than 64 levels keep the member's value). The plan holds its own copies (CSR,
 * traversal state, outputs of the widest request x the union's vertices), so
 * the graphs may be closed after create; one run at a time per plan. Apart
 * from alpha, a union runs with the batch options of its member with the most
 * edges. */
typedef struct ent_multi ent_multi;
int ent_multi_create(ent_graph* const* graphs, int32_t n_graphs, const int32_t* src,
                     const int32_t* n_src, ent_multi** out);
int ent_multi_run(ent_multi* plan, double* device_ms);
int ent_multi_depths(ent_multi* plan, int32_t k, int32_t* depth_out);
int ent_multi_destroy(ent_multi* plan);
/* Per-level trace of the union that holds graph k: one host-driven run of the
 * plan's kernels for that width class (its rows are then readable with
 * ent_multi_depths), one row per level and the final flush as level -1, as
 * ent_bfs_batch_trace writes them; *n_levels rows. */
int ent_multi_trace(ent_multi* plan, int32_t k, ent_level_trace* out, int32_t max_levels,
                    int32_t* n_levels);

/* ------------------------------------------------- several GPUs --------- */
/* Many sources over replicas of one graph on several GPUs of a node. No
 * reference counterpart (the reference drives one GPU, bfs_gpu_opt.cuh:305).
 * Sources are independent, so nothing is exchanged on the data path: the
 * source list is cut into contiguous chunks (ent_replicas_plan), one host
 * thread per replica takes the next unclaimed chunk and runs it as one bitwise
 * batch on its own GPU, and each chunk's rows land at the chunk's own rows of
 * the output, so results are in input order whichever replica ran a chunk.
 * Every kernel reads only its own replica; no peer memory is used. */
typedef struct ent_replicas ent_replicas;
/* Chunk boundaries for n_src sources over n_replicas: chunks of
 * min(max_batch, ceil(n_src / n_replicas)) sources, the last one shorter.
 * chunk_begin (may be NULL) receives *n_chunks + 1 entries: chunk c covers
 * sources [chunk_begin[c], chunk_begin[c+1]). Host-only arithmetic. */
int ent_replicas_plan(int32_t n_src, int32_t n_replicas, int32_t max_batch, int32_t* chunk_begin,
                      int32_t* n_chunks);
/* graphs: one handle per replica, the same graph (equal V and E) on the GPUs
 * of the caller's choice (borrowed: destroy them after the replica set).
 * Default max_batch 1024 sources per chunk. */
int ent_replicas_create(ent_graph* const* graphs, int32_t n_replicas, ent_replicas** out);
int ent_replicas_set_max_batch(ent_replicas* r, int32_t max_batch);
/* depth_out: HOST n_src x V int32 (row s = src[s]'s depths) or NULL; stats:
 * n_src entries or NULL. Same depths as ent_bfs_batch / n_src ent_bfs calls. */
int ent_replicas_bfs_batch(ent_replicas* r, const int32_t* src, int32_t n_src, int32_t* depth_out,
                           ent_stats* stats);
/* The same with the reference's byte depths (see ent_bfs_batch_u8). */
int ent_replicas_bfs_batch_u8(ent_replicas* r, const int32_t* src, int32_t n_src, uint8_t* depth_out,
                              ent_stats* stats);
/* Sources each replica ran in the last call (n_replicas entries). */
int ent_replicas_sources_run(const ent_replicas* r, int64_t* per_replica);
int ent_replicas_destroy(ent_replicas* r);

/* ------------------------------------------------------ autotuning ------ */
/* Coordinate-descent search of the traversal thresholds on this graph and
 * GPU (the reference fixes them at compile time: bfs_gpu_opt.cuh:323-324,
 * comm.h:155, comm.h:176-177, inspector.cuh:497). mode 0 tunes the
 * single-source knobs (tiers, chunk size, hub cache, alpha/beta, CTAs per SM)
 * timing ent_bfs over `src`; mode 1 tunes the batched knobs timing one
 * ent_bfs_batch of all of `src`. Every candidate gives the same depths. The
 * best options are applied to g and returned with their device time. */
int ent_autotune(ent_graph* g, const int32_t* src, int32_t n_src, int32_t mode, int32_t reps,
                 ent_bfs_opts* best, double* best_ms);

/* ------------------------------------------------------- serving -------- */
/* A request loop over device-resident graphs with continuous batching. No
 * reference counterpart (the reference runs a fixed 64-source list per
 * process). Each graph has slots_per_graph concurrent batched launches; a
 * scheduler thread forms each batch from the queries waiting at the moment a
 * slot frees up (at most max_batch, and only queries that get a depth row).
 * Per-query state is one depth row (V int32) in a per-graph HBM pool sized by
 * rows_per_graph or, when 0, by hbm_budget_bytes (0 = a quarter of free HBM):
 * a query holds its row from launch until ent_server_release, so unreleased
 * results throttle admission. submit fails with ENT_ERR_ADMISSION once
 * max_pending queries wait. Results are the same depths as ent_bfs.
 * High-diameter graphs (grids, road-like graphs) would keep a batch on the
 * device for thousands of levels: a graph whose probe traversal (run once at
 * creation from its first non-isolated vertex) has at least
 * single_source_levels levels is served one source per launch instead, by
 * single_slots concurrent single-source traversals (each runs its small
 * frontiers inside one thread-block cluster). */
typedef struct ent_server ent_server;
typedef struct ent_server_opts {
  int32_t max_batch;        /* sources per batched launch, 1..2048 (default 64) */
  int32_t slots_per_graph;  /* concurrent batches per graph, 1..16 (default 2)  */
  int32_t rows_per_graph;   /* depth rows per graph, 0 = from the budget         */
  int32_t max_pending;      /* waiting queries before submit refuses             */
  int64_t hbm_budget_bytes; /* depth-row budget across graphs, 0 = free HBM / 4  */
  int32_t single_source_levels; /* probe depth from which a graph is served one
                                   source per launch (default 64, 0 = never)    */
  int32_t single_slots;     /* concurrent single-source traversals per such graph,
                               1..64 (default 8)                                 */
  int32_t fast_slots;       /* single-source slots of every other graph, 0..16
                               (default 2, 0 = none): they take the graph's
                               queries while at most fast_max_waiting wait, where
                               one direction-optimising traversal per query beats
                               a bitwise batch of a few                          */
  int32_t fast_max_waiting; /* default 2                                          */
  int32_t single_cluster;   /* CTAs per small-frontier cluster of the deep graphs'
                               single-source slots, 0..16 (default 8; 0 = each
                               graph's own narrow_cluster option)                */
  int32_t join;             /* queries waiting while a batch of their graph runs
                               join it at a level boundary, in its free source
                               positions, while the batch is at level <= join
                               (default 1; 0 = never: they wait for a slot). A
                               batch's results come back when it ends, so joining
                               late would hold back the results already in it */
} ent_server_opts;
typedef struct ent_query_result {
  int64_t query_id;
  int32_t graph;
  int32_t src;
  int64_t reached_vertices;
  int64_t traversed_edges;
  int32_t levels;
  int32_t status;           /* 0 ok, else an ent_status */
  double latency_ms;        /* submit -> result on the device */
  double queue_ms;          /* submit -> launch */
} ent_query_result;
typedef struct ent_server_counters {
  int64_t submitted, rejected, completed, released, batches, launched, pending, rows_total, rows_free;
  int32_t max_batch_seen;
  int32_t single_graphs;    /* graphs served one source per launch */
  int64_t fast_launches;    /* queries run on the fast single-source slots of the other graphs */
  int64_t joined;           /* queries that joined a running batch at a level boundary */
} ent_server_counters;
void ent_server_opts_default(ent_server_opts* opts);
int ent_server_create(ent_graph* const* graphs, int32_t n_graphs, const ent_server_opts* opts,
                      ent_server** out);
int ent_server_submit(ent_server* s, int32_t graph, int32_t src, int64_t* query_id);
/* Completed queries (up to max_results); waits up to wait_us if none is ready.
 * A query's depths stay readable (ent_server_depth, _device) until it is
 * released, which frees its depth row for the next query. */
int ent_server_poll(ent_server* s, ent_query_result* out, int32_t max_results, int32_t* n_out,
                    int32_t wait_us);
int ent_server_depth(ent_server* s, int64_t query_id, int32_t* depth_out);
int ent_server_depth_device(ent_server* s, int64_t query_id, const int32_t** depth_dev);
int ent_server_release(ent_server* s, int64_t query_id);
int ent_server_get_counters(ent_server* s, ent_server_counters* out);
int ent_server_destroy(ent_server* s);

#ifdef __cplusplus
}
#endif
#endif /* ENTERPRISE_B200_H */
