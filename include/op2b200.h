/*
 * op2b200.h -- C-ABI of the B200 (sm_100a) PyOP2 backend library.
 *
 * Every entry point takes plain pointers, sizes and opaque uint64_t handles
 * (device pointers, streams, modules, plans, sparsities).  No torch or Python
 * types cross this boundary, so the library can be bound from ctypes (the
 * Python backend does this), cffi, or any FFI.
 *
 * All functions return OP2B_OK (0) on success or one of the OP2B_ERR_* codes;
 * op2b_last_error() returns the message of the last failure on the calling
 * thread.  Nothing in the library calls abort() or exit().
 *
 * Citations name the reference (gbts/PyOP2) interface each entry point
 * replaces, as path:line within that project.
 */
#ifndef OP2B200_H
#define OP2B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OP2B_OK            0
#define OP2B_ERR_CUDA      1   /* a CUDA runtime call failed              */
#define OP2B_ERR_NVRTC     2   /* JIT compilation of a par_loop stub      */
#define OP2B_ERR_ARG       3   /* invalid argument (size, handle, index)  */
#define OP2B_ERR_NOMEM     4   /* device or host allocation failed        */
#define OP2B_ERR_STATE     5   /* library not initialised / already shut  */
#define OP2B_ERR_MAP       6   /* a Map value lies outside its target Set */

/* ------------------------------------------------------------------------
 * Context.  Replaces cuda._setup (pyop2/cuda.py:824-847), which created one
 * PyCUDA context and stream and read WARP_SIZE / MAX_SHARED_MEMORY_PER_BLOCK,
 * and op2.exit (pyop2/op2.py:84-90).
 * ---------------------------------------------------------------------- */
int op2b_init(int device);
int op2b_shutdown(void);
int op2b_version(void);
int op2b_last_error(char *buf, size_t len);
/* sm_count, max opt-in dynamic shared memory per block, compute capability,
 * global memory bytes, L2 bytes. */
int op2b_device_info(int32_t *sm_count, int32_t *smem_optin, int32_t *cc_major,
                     int32_t *cc_minor, uint64_t *total_mem, uint64_t *l2_bytes);
/* Maximum L2 fetch granularity of this process's context (32, 64 or 128
 * bytes; a per-context limit, cudaLimitMaxL2FetchGranularity).  Indirect
 * gathers of Dat rows of 8-32 bytes through permuted Maps fetch less unused
 * data at 32.  No reference counterpart (PyCUDA used the default). */
int op2b_set_l2_fetch_granularity(int32_t bytes);

/* ------------------------------------------------------------------------
 * Device memory and transfers.  Replaces the PyCUDA gpuarray allocations and
 * set()/get() used by DeviceDataMixin._allocate_device/_to_device/_from_device
 * (pyop2/cuda.py:133-153) and Map._to_device (pyop2/cuda.py:375-388).
 * Allocation is stream-ordered (no device-wide synchronisation on free).
 * ---------------------------------------------------------------------- */
int op2b_malloc(uint64_t *dptr, uint64_t bytes);
int op2b_free(uint64_t dptr);
int op2b_host_alloc(uint64_t *hptr, uint64_t bytes);   /* pinned host memory */
int op2b_host_free(uint64_t hptr);
int op2b_memcpy_h2d(uint64_t dst, const void *src, uint64_t bytes, uint64_t stream);
int op2b_memcpy_d2h(void *dst, uint64_t src, uint64_t bytes, uint64_t stream);
/* Host-to-device copy of at most 256 bytes carried in the launch parameters
 * of a one-block kernel: asynchronous from any host memory (the bytes are
 * captured at the call), so uploading a Global's value never waits for the
 * stream as a pageable-memory copy does.  No reference counterpart (PyCUDA
 * copied Globals with synchronous memcpy_htod, pyop2/cuda.py:325-340). */
int op2b_memcpy_h2d_small(uint64_t dst, const void *src, uint64_t bytes, uint64_t stream);
/* Device-to-host copy that returns at once (stream-ordered; complete when an
 * event recorded after it completes).  dst must be pinned host memory
 * (op2b_host_alloc) for the copy to be asynchronous. */
int op2b_memcpy_d2h_async(void *dst, uint64_t src, uint64_t bytes, uint64_t stream);
int op2b_memcpy_d2d(uint64_t dst, uint64_t src, uint64_t bytes, uint64_t stream);
int op2b_memset(uint64_t dst, int value, uint64_t bytes, uint64_t stream);
/* AoS <-> SoA reorder on the device, [n][dim] <-> [dim][n] with elements of
 * elem_bytes (1,2,4,8).  Replaces DeviceDataMixin._maybe_to_soa/_maybe_to_aos
 * (pyop2/device.py:153-174), which transposed on the host. */
int op2b_transpose(uint64_t dst, uint64_t src, int64_t n, int32_t dim,
                   int32_t elem_bytes, int32_t to_soa, uint64_t stream);
/* Check that every value of a Map lies in [0, to_size); returns OP2B_ERR_MAP
 * with the first offending position otherwise.  The reference trusted Map
 * values (pyop2/base.py:1040-1048); out-of-range values would make a device
 * kernel read outside a Dat. */
int op2b_map_validate(uint64_t map, int64_t n_values, int32_t to_size,
                      int64_t *bad_index, uint64_t stream);

/* ------------------------------------------------------------------------
 * Streams, events, CUDA graphs.  The reference used a single stream and
 * synchronised after every par_loop (pyop2/cuda.py:656-658).  stream == 0
 * names the library's own default op2 stream.
 * ---------------------------------------------------------------------- */
int op2b_default_stream(uint64_t *stream);
int op2b_stream_create(uint64_t *stream);
int op2b_stream_destroy(uint64_t stream);
int op2b_stream_sync(uint64_t stream);
int op2b_device_sync(void);
int op2b_event_create(uint64_t *event);
int op2b_event_destroy(uint64_t event);
int op2b_event_record(uint64_t event, uint64_t stream);
/* As op2b_event_record, but while the stream is being captured into a CUDA
 * graph the record becomes a node of the graph, so every replay records the
 * event (device timestamps inside a replayed graph). */
int op2b_event_record_node(uint64_t event, uint64_t stream);
int op2b_event_sync(uint64_t event);
/* Non-blocking: *done = 1 if all work before the event's record has
 * completed, else 0 (cudaEventQuery). */
int op2b_event_query(uint64_t event, int32_t *done);
int op2b_event_elapsed_ms(uint64_t start, uint64_t stop, float *ms);
int op2b_stream_wait_event(uint64_t stream, uint64_t event);
int op2b_graph_begin(uint64_t stream);
int op2b_graph_end(uint64_t stream, uint64_t *graph_exec);
int op2b_graph_launch(uint64_t graph_exec, uint64_t stream);
int op2b_graph_destroy(uint64_t graph_exec);
/* Overlapped capture (no direct reference counterpart: the reference ran
 * every par_loop in program order on one stream).  A capture on one stream
 * records a linear chain of nodes.  op2b_graph_capture_tail returns the
 * chain's last node so far (0 before the first); op2b_graph_end_capture ends
 * the capture and returns the un-instantiated graph; op2b_graph_chain_positions
 * gives each marked node's position on the chain (-1 for a 0 mark) and the
 * chain length; op2b_graph_relax takes segments [seg_first[s], seg_last[s]]
 * that tile the chain in order and, for each segment s > 0, replaces the chain
 * edge into its first node by edges from the last nodes of the earlier
 * segments dep_idx[dep_ptr[s] .. dep_ptr[s+1]), then instantiates the graph
 * (nseg == 0: instantiate unchanged).  The graph stays owned by the caller:
 * free it with op2b_graph_free. */
int op2b_graph_capture_tail(uint64_t stream, uint64_t *node);
int op2b_graph_end_capture(uint64_t stream, uint64_t *graph);
int op2b_graph_chain_positions(uint64_t graph, const uint64_t *marks, int32_t nmarks,
                               int64_t *pos, int64_t *nnodes);
int op2b_graph_relax(uint64_t graph, const int64_t *seg_first, const int64_t *seg_last,
                     int32_t nseg, const int32_t *dep_ptr, const int32_t *dep_idx,
                     uint64_t *graph_exec);
int op2b_graph_free(uint64_t graph);

/* ------------------------------------------------------------------------
 * JIT modules.  Replaces cuda.JITModule.compile (pyop2/cuda.py:610-651):
 * PyCUDA SourceModule + Const upload.  The source is compiled by NVRTC for
 * sm_100a straight to a cubin, which the caller may cache and reload.
 * ---------------------------------------------------------------------- */
int op2b_nvrtc_compile(const char *src, const char *name, const char *const *opts,
                       int32_t nopts, void **cubin, uint64_t *cubin_bytes,
                       char *log, uint64_t log_len);
int op2b_cubin_free(void *cubin);
int op2b_module_load(const void *cubin, uint64_t *module);
int op2b_module_unload(uint64_t module);
int op2b_module_function(uint64_t module, const char *name, uint64_t *fn);
/* Device address and size of a __constant__ / __device__ symbol of a module
 * (Const._to_device, pyop2/cuda.py:314-320). */
int op2b_module_global(uint64_t module, const char *name, uint64_t *dptr, uint64_t *bytes);
int op2b_function_set_smem(uint64_t fn, int32_t bytes);
/* Resident CTAs per SM of fn at the given block size and dynamic shared
 * memory, for sizing persistent grids (batched loops).  No reference
 * counterpart (the reference launched one CTA per plan block). */
int op2b_function_occupancy(uint64_t fn, uint32_t block, uint32_t smem, int32_t *blocks_per_sm);
/* Launch fn with ONE by-value parameter: the packed struct params[0..nbytes).
 * The generated stubs all take a single struct argument. */
int op2b_launch(uint64_t fn, uint32_t grid, uint32_t block, uint32_t smem,
                uint64_t stream, const void *params, uint64_t nbytes);
/* on != 0: op2b_launch and op2b_launch_colored launch with programmatic
 * stream serialisation, so a stub's CTAs may be scheduled while the kernel
 * before it on the stream finishes; the generated stubs wait for that
 * kernel's completion (griddepcontrol.wait) before touching memory, so
 * results are unchanged.  Only for functions of generated stubs.  No
 * reference counterpart (the reference synchronised the host after every
 * par_loop, pyop2/cuda.py:656-658). */
int op2b_set_programmatic_launch(int32_t on);
/* Colour-by-colour launch of an indirect stub: for colour c the int32 pair at
 * params+col_field_offset is set to (first block of c, blocks in c) and the
 * stub is launched on grid = blocks in c.  Replaces the per-colour host loop
 * with a stream synchronise before each launch (pyop2/cuda.py:757-800). */
int op2b_launch_colored(uint64_t fn, int32_t ncolors, const int32_t *ncolblk,
                        uint32_t block, uint32_t smem, uint64_t stream,
                        void *params, uint64_t nbytes, uint64_t col_field_offset);

/* ------------------------------------------------------------------------
 * Plan: partitioning, staging maps and conflict colouring, built on the GPU.
 * Replaces plan.pyx Plan.__cinit__ (pyop2/plan.pyx:93-376) and the cached
 * _GenericPlan (pyop2/device.py:257-322).
 *
 * Staging pairs (one per unique indirect (Dat, Map)): stage_map[s] device map
 * [set_size][stage_arity[s]], stage_nidx[s] indices taken from
 * stage_idx[stage_idx_off[s] ...], stage_bytes[s] = itemsize*cdim of the Dat.
 * Race groups (one per Dat written with INC, or Mat row set when matrix
 * colouring is on): race_nent[g] (map, idx) entries taken from the flat
 * race_map/race_arity/race_idx arrays, target Set size race_size[g].
 * flags: bit0 staging, bit1 thread colouring.
 * ---------------------------------------------------------------------- */
#define OP2B_PLAN_STAGING         1
#define OP2B_PLAN_THREAD_COLORING 2

int op2b_plan_build(int32_t set_size, int32_t part_size,
                    int32_t nstage, const uint64_t *stage_map, const int32_t *stage_arity,
                    const int32_t *stage_nidx, const int32_t *stage_idx_off,
                    const int32_t *stage_idx, const int32_t *stage_bytes,
                    int32_t nrace, const int32_t *race_nent, const int32_t *race_size,
                    const uint64_t *race_map, const int32_t *race_arity,
                    const int32_t *race_idx, int32_t flags, uint64_t stream,
                    uint64_t *plan);
/* Scalars: nblocks, ncolors, nshared (max staged bytes per block, 16-byte
 * aligned per pair), ninds (unique staging pairs), max_nthrcol,
 * total staged ind_map length, loc_map rows. */
int op2b_plan_info(uint64_t plan, int32_t *nblocks, int32_t *ncolors, int32_t *nshared,
                   int32_t *ninds, int32_t *max_nthrcol, int64_t *ind_map_len,
                   int32_t *loc_rows);
/* Device arrays of the plan, in the reference layout (plan.pyx:140-212,
 * 274-376):  0 nelems, 1 offset, 2 ind_map, 3 loc_map (int16), 4 ind_sizes,
 * 5 ind_offs, 6 nindirect, 7 thrcol, 8 nthrcol, 9 blkmap, 10 ncolblk, and
 * 11 blkcol (colour of every block). */
int op2b_plan_array(uint64_t plan, int32_t which, uint64_t *dptr, int64_t *count);
/* Host copy of ncolblk (ncolors entries), used to launch colour by colour. */
int op2b_plan_ncolblk_host(uint64_t plan, int32_t *out, int32_t n);
int op2b_plan_free(uint64_t plan);

/* ------------------------------------------------------------------------
 * Locality partition for staged indirect loops.  The reference partitions
 * into blocks of consecutive elements (pyop2/plan.pyx:107-110) and stages
 * each block's indirect rows in shared memory (:112-212); on a permuted mesh
 * numbering consecutive elements share no targets, so this builder first
 * reorders the iteration set into compact regions: seeds hashed from
 * element ids (about one per region_size elements), a multi-source
 * breadth-first search over the element graph of grow_map (elements sharing
 * a target are adjacent; ties to the smaller region id, so the result is
 * deterministic), elements sorted by (region, level, id), each region cut
 * into nearly equal blocks of at most part_size elements.  Then, per block
 * and staged Map (all rows), the sorted distinct targets and, per position
 * of the reordered set and Map row, the target's index among them; and per
 * block the reference's greedy thread colouring (pyop2/plan.pyx:282-324)
 * over the targets of the staged Maps with stage_inc[s] != 0, so elements of
 * one colour never share such a target.  part_size * stage_arity must not
 * exceed 16384; at most 64 staged Maps.
 * ---------------------------------------------------------------------- */
int op2b_region_plan_build(int32_t set_size, int32_t part_size, int32_t region_size,
                           uint64_t grow_map, int32_t grow_arity, int32_t grow_ntargets,
                           int32_t nstage, const uint64_t *stage_map, const int32_t *stage_arity,
                           const int32_t *stage_inc, uint64_t stream, uint64_t *plan);
/* max_count: nstage entries, the largest distinct-target count of a block;
 * max_nthrcol: the most thread colours of a block. */
int op2b_region_plan_info(uint64_t plan, int32_t *nblocks, int32_t *nregions, int32_t *levels,
                          int32_t *max_count, int64_t *tlist_len, int32_t *max_nthrcol);
/* Device arrays (int32 unless noted): 0 order [set_size] (element at each
 * position), 1 boff [nblocks+1] (first position of each block), 2 tlist
 * (distinct targets, block-major then staged Map), 3 toff [nblocks*nstage+1]
 * (offset of each (block, Map) list in tlist), 4 tcnt [nblocks*nstage],
 * 5 loc (int16) [sum of arities][set_size]: row r of staged Map s for the
 * element at position pos is tlist[toff[b*nstage+s] + loc[(row0(s)+r)*set_size+pos]],
 * 6 thrcol [set_size] (thread colour per position), 7 nthrcol [nblocks]. */
int op2b_region_plan_array(uint64_t plan, int32_t which, uint64_t *dptr, int64_t *count);
/* Renumber a built plan's staged slots so that the rows eight consecutive
 * positions of a block read (one quarter-warp of a staged stub, for any CTA
 * size) lie in distinct 16-byte shared-memory bank groups where the targets
 * allow: per (block, staged Map) a greedy choice of slot residue mod 8 over
 * the groups of 8 positions, row by row, then slots grouped by residue.  A
 * block's slot count becomes 8 x its largest residue class; padding slots
 * have target -1 in tlist (stubs skip them).  tcnt, toff, tlist, loc and the
 * max counts of op2b_region_plan_info change; order, boff and the colours
 * do not.  Idempotent.  No reference counterpart (the reference staged rows
 * in sorted target order, pyop2/plan.pyx:112-212). */
int op2b_region_plan_bank_slots(uint64_t plan, uint64_t stream);
int op2b_region_plan_free(uint64_t plan);

/* ------------------------------------------------------------------------
 * Sparsity: CSR pattern built on the GPU.  Replaces core.build_sparsity
 * (pyop2/op_lib_core.pyx:544-596) and build_sparsity_pattern_seq
 * (pyop2/sparsity_utils.cxx:5-51): rows = rmult*rmap+r, cols = cmult*cmap+c,
 * union over all map pairs, colidx sorted within each row.
 * iterset_size[m] is the element count of pair m (its row map's from-set).
 * ---------------------------------------------------------------------- */
int op2b_sparsity_build(int32_t rmult, int32_t cmult, int32_t nrows, int32_t ncols,
                        int32_t nmaps, const uint64_t *rmaps, const int32_t *rarity,
                        const uint64_t *cmaps, const int32_t *carity,
                        const int32_t *iterset_size, uint64_t stream, uint64_t *sparsity);
/* lsize = nrows*rmult rows; nz = number of stored entries. */
int op2b_sparsity_info(uint64_t sparsity, int32_t *lsize, int64_t *nz);
/* Device arrays: rowptr (lsize+1 int32), colidx (nz int32), nnz (lsize int32). */
int op2b_sparsity_arrays(uint64_t sparsity, uint64_t *rowptr, uint64_t *colidx,
                         uint64_t *nnz);
int op2b_sparsity_free(uint64_t sparsity);

/* ------------------------------------------------------------------------
 * Incidence: for each target t of a Map [nelem][arity] (values in
 * [0, ntargets)), the flat positions e*arity+k with map[e*arity+k] == t, sorted
 * ascending (element order, then map index).  Owner-computes stubs use it to
 * add all contributions to one target in the order the sequential backend
 * adds them (pyop2/sequential.py:55-72).  No direct reference counterpart:
 * it replaces the LMA buffer + atomic scatter of pyop2/cuda.py:177-270 and
 * the coloured INC of cuda_indirect_loop.jinja2:169-189 for those loops.
 * ---------------------------------------------------------------------- */
int op2b_incidence_build(uint64_t map, int32_t nelem, int32_t arity, int32_t ntargets,
                         uint64_t stream, uint64_t *incidence);
/* ptr: ntargets+1 int32 offsets; list: nelem*arity int32 flat positions. */
int op2b_incidence_arrays(uint64_t incidence, uint64_t *ptr, uint64_t *list,
                          int32_t *max_degree);
int op2b_incidence_free(uint64_t incidence);
/* Targets of a Map [nelem][arity] in order of first use along an element
 * order: position q = pos*arity + k stands for row k of element
 * elem_order[pos] (elem_order 0: element pos); target_order receives the
 * ntargets ids sorted by their smallest q, targets no element uses last in
 * increasing id.  The thread-per-target gather stubs walk targets in this
 * order so that neighbouring threads gather neighbouring rows.  No direct
 * reference counterpart (the reference walks elements in set order,
 * pyop2/plan.pyx:107-110). */
int op2b_first_use_order(uint64_t map, int32_t arity, int64_t nelem, uint64_t elem_order,
                         int32_t ntargets, uint64_t target_order, uint64_t stream);
/* READ replicas in first-use order.  dst row i = src row index[i] (n rows of
 * row_bytes, a multiple of 4); and dst_map[q] = r where order[r] ==
 * map[q] (order a permutation of [0, ntargets)).  With order from
 * op2b_first_use_order, a loop that only reads a Dat through a Map reads a
 * copy of the Dat in order of first use through the renumbered Map: rows
 * that neighbouring elements read lie next to each other.  No direct
 * reference counterpart (the reference gathers through the user's
 * numbering, pyop2/assets/cuda_indirect_loop.jinja2:105-150). */
int op2b_rows_gather(uint64_t dst, uint64_t src, uint64_t index, int64_t n, int32_t row_bytes,
                     uint64_t stream);
int op2b_map_renumber(uint64_t dst_map, uint64_t map, int64_t n_entries, uint64_t order,
                      int32_t ntargets, uint64_t stream);

/* ------------------------------------------------------------------------
 * Halo rows of partitioned sets.  Replaces the host-side packing of
 * Dat.halo_exchange_begin / _end (pyop2/base.py:797-835:
 * send_buf = data[sends[dest]]; data[receives[source]] = recv_buf).
 * op2b_halo_pack: buf[i] = rows[index[i]]; op2b_halo_unpack:
 * rows[index[i]] = buf[i]; n rows of row_bytes bytes each, index int32.
 * ---------------------------------------------------------------------- */
int op2b_halo_pack(uint64_t buf, uint64_t rows, uint64_t index, int64_t n, int32_t row_bytes,
                   uint64_t stream);
int op2b_halo_unpack(uint64_t rows, uint64_t buf, uint64_t index, int64_t n, int32_t row_bytes,
                     uint64_t stream);

/* ------------------------------------------------------------------------
 * Two-phase deterministic INC.  A generated stub writes every element's INC
 * contribution to a tiled contribution array: element e, position k (of K)
 * at row ((e / 32) * K + k) * 32 + e % 32, cdim values per row (k: map
 * position of a Dat INC, or r * ca + c of a Mat's local entry);
 * op2b_lma_reduce then adds, for each target t, the contributions listed by
 * t's incidence (increasing element order) to out[t] in that order -- the
 * order pyop2/sequential.py:55-72 adds them -- optionally with compensated
 * (Kahan) summation.  out and lma are float64.  Replaces the LMA buffer +
 * atomic scatter of pyop2/cuda.py:177-270 and the coloured INC of
 * cuda_indirect_loop.jinja2:169-189 where the result must not depend on
 * scheduling.
 * ---------------------------------------------------------------------- */
/* Incidence of a scalar Mat assembly over CSR positions: for each position,
 * the local entries that add to it, in element order, each given as its
 * index in the tiled contribution array (K = ra * ca).  Fails with
 * OP2B_ERR_MAP if an entry is not in the Sparsity. */
int op2b_mat_incidence_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap, uint64_t cmap,
                             int32_t nelem, int32_t ra, int32_t ca, int32_t nnz,
                             uint64_t stream, uint64_t *incidence);
/* flags: OP2B_LMA_KAHAN compensated sums; OP2B_LMA_FROM_ZERO start from 0
 * instead of reading out[] (the caller knows the target is zero);
 * OP2B_LMA_MAT_INDEX the incidence comes from op2b_mat_incidence_build
 * (list entries are contribution-array indices; cdim 1, arity and kmask
 * ignored).  Otherwise the incidence is a Map's (op2b_incidence_build: flat
 * positions e * arity + k), positions whose k is not set in kmask are
 * skipped, cdim is 1 to 4 and arity at most 64. */
#define OP2B_LMA_KAHAN     1
#define OP2B_LMA_FROM_ZERO 2
#define OP2B_LMA_MAT_INDEX 4
int op2b_lma_reduce(uint64_t out, int32_t cdim, uint64_t ptr, uint64_t list, int32_t ntargets,
                    uint64_t lma, int64_t nelem, int32_t arity, uint64_t kmask, int32_t flags,
                    uint64_t stream);

/* ------------------------------------------------------------------------
 * Linear algebra on device CSR Mats (float64 values, int32 rowptr/colidx)
 * and Dat vectors.  Replaces the PETSc KSP solve of pyop2/petsc_base.py:
 * 160-220 (defaults 'cg' + 'jacobi', pyop2/base.py:1591-1601), the Cusp CG of
 * pyop2/cuda.py:445-600, and the host-side Dat arithmetic and norm of
 * pyop2/base.py:749-797, 836-839.  Reductions are deterministic (fixed
 * combination order for a given launch shape).
 * ---------------------------------------------------------------------- */
/* y = alpha * A x + beta * y over nrows rows (beta == 0: y is not read).
 * group: lanes per row (1, 2, 4, 8, 16 or 32; 0 picks by the mean row length). */
int op2b_csr_spmv(uint64_t rowptr, uint64_t colidx, uint64_t vals, int32_t nrows, int64_t nnz,
                  uint64_t x, uint64_t y, double alpha, double beta, int32_t group,
                  uint64_t stream);
/* out[i] = x[i] op y[i] (y != 0) or x[i] op yscalar (y == 0); op 0 add,
 * 1 subtract, 2 multiply, 3 divide; dtype 0 float64, 1 float32, 2 int32;
 * out may equal x. */
int op2b_vec_binop(uint64_t out, uint64_t x, uint64_t y, double yscalar, int64_t n, int32_t op,
                   int32_t dtype, uint64_t stream);
/* *result = sum_i x[i] * y[i] (float64), returned to the host. */
int op2b_vec_dot(uint64_t x, uint64_t y, int64_t n, double *result, uint64_t stream);
/* Conjugate gradients on A x = b from x = 0, left-preconditioned by the
 * inverse diagonal of A (jacobi != 0) or not.  Stops at the first iteration
 * k whose preconditioned residual norm r_k = ||M^-1 (b - A x_k)|| satisfies
 * r_k <= max(rtol * r_0, atol) (reason 1), r_k >= dtol * r_0 (reason 2), is
 * not finite (reason 3), or at k = max_it (reason 4).  iterations = k;
 * history (may be NULL) receives r_0 .. r_k (iterations + 1 values). */
int op2b_cg_solve(uint64_t rowptr, uint64_t colidx, uint64_t vals, int32_t nrows, int64_t nnz,
                  uint64_t x, uint64_t b, int32_t jacobi, double rtol, double atol, double dtol,
                  int32_t max_it, int32_t *iterations, int32_t *reason, double *history,
                  uint64_t stream);

/* ------------------------------------------------------------------------
 * Mat operations on the device CSR values (dtype 4 = float32, 8 = float64).
 * Replaces cuda.Mat.zero_rows / zero (pyop2/cuda.py:289-301) and PETSc
 * MatZeroRowsLocal (pyop2/petsc_base.py:131-135).
 * ---------------------------------------------------------------------- */
/* Every stored entry of rows[0 .. nrows_zero) becomes 0 and each row's
 * diagonal entry, where the pattern stores one, becomes diag.  mat_rows is
 * the CSR's row count (rowptr holds mat_rows + 1 entries): a listed row
 * outside [0, mat_rows), or elem_bytes other than 4 or 8, is rejected with
 * OP2B_ERR_ARG before anything is allocated, copied or launched. */
int op2b_mat_zero_rows(uint64_t vals, uint64_t rowptr, uint64_t colidx, int32_t mat_rows,
                       const int32_t *rows, int32_t nrows_zero, double diag,
                       int32_t elem_bytes, uint64_t stream);

/* Scatter-slot table of a scalar Mat assembled through the Map pair
 * (rmap [nelem][ra], cmap [nelem][ca]): slots[(r*ca + c)*nelem + e] is the
 * CSR position of (rmap[e][r], cmap[e][c]), or -1 where the Sparsity has no
 * such entry.  slots holds nelem*ra*ca int32.  The assembly stubs read it
 * instead of searching the row for every entry.  No direct reference
 * counterpart: it replaces the per-entry row search of the LMA-to-CSR scatter
 * (assets/cuda_matrix_support.jinja2:27-81) and PETSc's MatSetValues lookup. */
int op2b_mat_slots_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap, uint64_t cmap,
                         int64_t nelem, int32_t ra, int32_t ca, uint64_t slots, uint64_t stream);
/* Compact form of the same table: slots[r*nelem + e] (uint64) holds in byte
 * c the position of (rmap[e][r], cmap[e][c]) counted from rowptr[rmap[e][r]]
 * (255 where the Sparsity has no such entry); ca <= 8, and rows of at most
 * 254 stored entries.  8 bytes per (element, local row) instead of 4 per
 * local entry; the stubs add the row start they read through the Map.  No
 * direct reference counterpart (see op2b_mat_slots_build). */
int op2b_mat_slots_rel_build(uint64_t rowptr, uint64_t colidx, uint64_t rmap, uint64_t cmap,
                             int64_t nelem, int32_t ra, int32_t ca, uint64_t slots,
                             uint64_t stream);
/* op2b_mat_zero_rows for callers that must not allocate device memory.
 * No counterpart in the reference.
 *
 * op2b_mat_zero_rows copies the row list to device memory it allocates (from
 * the stream-ordered pool) on every call.  Some callers cannot let the library
 * allocate: a solver loop that applies boundary conditions every time step
 * inside a process whose device memory is reserved up front by its host
 * framework (a further cudaMalloc fails or is forbidden there), or code that
 * must not risk the synchronisation or out-of-memory failure an allocation can
 * bring in the middle of a time step.  This entry point takes the same inputs
 * and outputs and allocates nothing: the row list goes into a fixed scratch
 * array compiled into the library (OP2B_ZERO_ROWS_STATIC_MAX rows, 256 KiB,
 * held on every GPU that loads the library until the process exits).
 *  - More than OP2B_ZERO_ROWS_STATIC_MAX rows is rejected with OP2B_ERR_ARG
 *    (split the list, or call op2b_mat_zero_rows); so are rows outside
 *    [0, mat_rows) and elem_bytes other than 4 or 8, before any copy or launch.
 *  - The first call on a device looks up the scratch array's device address
 *    (cudaGetSymbolAddress).
 *  - All calls share the one scratch array, which keeps the last call's row
 *    list: calls that overlap on the GPU (other streams, other threads) race
 *    and must be serialised by the caller.  The call returns after its work
 *    has finished on the stream (it synchronises the stream), so it cannot
 *    be recorded into a CUDA graph: call it outside any stream capture. */
#define OP2B_ZERO_ROWS_STATIC_MAX 65536
int op2b_mat_zero_rows_static(uint64_t vals, uint64_t rowptr, uint64_t colidx, int32_t mat_rows,
                              const int32_t *rows, int32_t nrows_zero, double diag,
                              int32_t elem_bytes, uint64_t stream);

#ifdef __cplusplus
}
#endif
#endif /* OP2B200_H */
