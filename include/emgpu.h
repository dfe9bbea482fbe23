/*
 * emgpu -- B200 (sm_100a) Nedelec-2 curl-curl assembly, C ABI.
 *
 * The drop-in replaces this part of EMerge (biruichen/EMerge v2.8.0):
 *
 *   Evec, Bvec, cscmap = tet_mass_stiffness_matrices(field, er, ur, conductor_tets, cscmap)
 *                                              physics/microwave/assembly/curlcurl.py:222-270
 *   A = cscmap.to_csc(Evec - Bvec * k0**2)     physics/microwave/assembly/assembler.py:494
 *                                              mth/csc_cast.py:51-63, 65-177
 *
 * Conventions
 * - Every pointer named d_* is DEVICE memory allocated by the caller (for
 *   example a torch tensor). The library never allocates or frees caller
 *   memory. Host pointers are named h_*.
 * - Arrays use the reference's layouts, C-contiguous: nodes f64[3][nN],
 *   tets i32[4][nT], tet_to_edge i32[6][nT], tet_to_tri i32[4][nT];
 *   material tensors in the compact layout of their kind (emg_material).
 * - Complex numbers are interleaved (re, im) pairs of double (complex128) or
 *   float (complex64).
 * - Every function returns 0 on success or a negative EMG_E* code; the
 *   message of the last failure in the calling thread is emg_last_error().
 *   No C++ exception crosses this boundary. Kernels never trap: index,
 *   orientation and capacity violations set bits in a caller-owned device
 *   status word (int64[2]: flags, first offending index), read with
 *   emg_status_read.
 * - All launches are ordered on the caller's stream; functions that must
 *   return a size synchronise that stream and say so.
 */
#ifndef EMGPU_H
#define EMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *emg_stream_t; /* a cudaStream_t; NULL = legacy default stream */

enum {
  EMG_OK = 0,
  EMG_EINVAL = -1,   /* bad argument (null pointer, size, enum) */
  EMG_ECUDA = -2,    /* a CUDA runtime call failed */
  EMG_EMESH = -3,    /* the device status word reports a bad mesh */
  EMG_ERANGE = -4,   /* a size exceeds what this build supports (e.g. nnz >= 2^31) */
  EMG_EDEVICE = -5,  /* no sm_100 device / kernel image not loadable */
};

/* status flags (device status word [0]) */
enum {
  EMG_ST_INDEX = 1,      /* a tet/edge/tri index outside its array */
  EMG_ST_DEGENERATE = 2, /* zero-volume / non-finite tet or repeated vertex */
  EMG_ST_CAPACITY = 4,   /* an entity exceeds a per-column capacity limit */
};

/* material kinds and the device layout of er / ur (complex128, per tet t of
 * the mesh, not of the assembled subset); ur may be NULL (identity) */
enum {
  EMG_MAT_ISO = 0,  /* scalars: er[t]                               (16 B/tet) */
  EMG_MAT_DIAG = 1, /* diagonals: er[d][t], d = 0..2                (48 B/tet) */
  EMG_MAT_FULL = 2, /* full tensors, the reference's er[r][c][t]   (144 B/tet) */
};

/* element value precision / form */
enum {
  EMG_FP64 = 0,  /* plain: the reference's arithmetic in FP64 (its absolute-
                    coordinate barycentric coefficients, KEAST4 points and
                    barycentric values, unfused), quadrature sums evaluated
                    as per-tet moments; element values complex128 */
  EMG_MIXED = 1, /* FP64 geometry (edge vectors, determinant, gradients,
                    orientation sign), FP64 tensors rounded to FP32 and
                    contracted in FP32 with FP32 accumulation against the
                    11-point rule's sums of basis products (exact for this
                    element, so precomputed); FP64 final sum; element
                    values complex64 */
  EMG_EXACT = 2, /* exact closed-form integrals on edge-vector geometry in
                    FP64 (free of the reference's cancellation error, so it
                    differs from the reference by that error); complex128 */
};

/* which element values a launch produces */
enum {
  EMG_OUT_LINCOMB = 0, /* one array: alpha*K_e + beta*M_e */
  EMG_OUT_K = 1,       /* stiffness (the reference's "dataE") */
  EMG_OUT_M = 2,       /* mass      (the reference's "dataB") */
};

/* element-value layouts */
enum {
  EMG_LAYOUT_COO = 0,    /* the reference's COO block: value[ia*400 + 20*a + b], a, b
                            reference DoF slots (curlcurl.py:449-455); symmetric */
  EMG_LAYOUT_PACKED = 1, /* upper triangle in the canonical (vertex-rank) DoF frame:
                            value[ia*210 + x*(41-x)/2 + (y-x)], x <= y; the
                            assembly path's layout (each unique entry computed
                            once, half the bytes) */
  EMG_LAYOUT_COO_T = 2,  /* D x D blocks per tet, transposed: value (i, j) of tet t
                            at D^2 t + D j + i (the Lagrange-2 element values
                            read by the COO gather with block_dofs = D) */
  EMG_LAYOUT_BLOCK = 3,  /* entity-pair blocks in the canonical frame: for the
                            tet's 10 entities (0-5 edges, 6-9 faces) and each
                            pair i <= j, the 2x2 values of their first and
                            second DoFs [(i1,j1), (i1,j2), (i2,j1), (i2,j2)]
                            at value[ia*220 + 4*(i*(21-i)/2 + j-i) + k]
                            (i1 = i, i2 = i+6 for edges; 12+i-6, 16+i-6 for
                            faces): one gather record and one 64-byte read
                            (32 for complex64) serve four entries of A */
};

typedef struct {
  int kind;          /* EMG_MAT_* */
  const void *d_er;  /* complex128, layout of `kind`, required */
  const void *d_ur;  /* complex128, layout of `kind`, or NULL (identity) */
} emg_material;

/* Gather plan: the sparsity pattern of A plus the element-slot -> nonzero map
 * of the column gather, stored in ONE caller-allocated device blob. Filled by
 * emg_plan_init (sizes, offsets) and emg_plan_build / emg_plan_finish. */
typedef struct {
  int64_t n_tets;    /* tets in the mesh */
  int64_t n_assy;    /* assembled tets (tetids length) */
  int64_t n_edges, n_tris;
  int64_t n_ent;     /* n_edges + n_tris: the column owners */
  int64_t n_items;   /* 10 * n_assy (entity, tet) incidences */
  int64_t N;         /* 2 * n_edges + 2 * n_tris */
  int64_t nnz;       /* set by emg_plan_build */
  int64_t max_col;   /* longest column, set by emg_plan_build */
  size_t off_ent_ptr, off_item, off_item_pos, off_ent_cnt; /* byte offsets in the blob */
  size_t off_contrib, off_posoff, off_pidx; /* gather lists: per output position of
                                     every entity chunk, its contributions as
                                     (item, row) and as packed value indices */
  size_t off_order;       /* int32 per entity chunk: the gather's processing order */
  size_t plan_bytes;      /* blob size */
  size_t workspace_bytes; /* scratch needed by emg_plan_build and emg_plan_order */
  int32_t record_bytes;   /* 8 (default) or 4: bytes per contribution record of the packed gather */
  int32_t value_layout;   /* EMG_LAYOUT_PACKED (default) or EMG_LAYOUT_BLOCK: the element values
                             emg_assemble writes and its gather reads */
  size_t off_hoff;        /* block layout: uint16 list start per row pair of every chunk */
} emg_plan;

int emg_version(void);
const char *emg_last_error(void);

/* Checks that `device` is an sm_100 GPU and that this library's kernels load
 * on it. Replaces nothing in the reference (it has no GPU path). */
int emg_device_check(int device);

/* Host-only, multi-threaded: the material kind of a complex128 [3][3][nT]
 * tensor array h_t (host memory, C order; the reference's er / ur layout,
 * curlcurl.py:222-235) -- EMG_MAT_FULL if any off-diagonal entry is nonzero,
 * else EMG_MAT_ISO if the three diagonals agree tet by tet, else EMG_MAT_DIAG --
 * and whether it is the identity (*h_identity = 1). n_threads <= 0: all host
 * threads. Lets the caller upload only the compact layout of emg_material. */
int emg_material_classify(const double *h_t, int64_t n_tets, int n_threads, int *h_kind, int *h_identity);

/* Status word helpers (d_status: int64[2] device memory). */
int emg_status_reset(int64_t *d_status, emg_stream_t stream);
int emg_status_read(const int64_t *d_status, int64_t *h_flags, int64_t *h_first_index, emg_stream_t stream);

/* Host-only: sizes and blob offsets for a mesh. Replaces the allocation part
 * of CSCMapping.from_rowcol (csc_cast.py:51-53). */
int emg_plan_init(int64_t n_tets, int64_t n_assy, int64_t n_edges, int64_t n_tris, emg_plan *plan);

/* Host-only, between emg_plan_init and emg_plan_build: the width of the
 * packed gather's per-contribution record. 8 bytes (default) store both value
 * indices; 4 bytes store the first and a bit, the second is derived on chip
 * (at most 10,226,078 assembled tets). 4 bytes halve that stream and the
 * plan's largest part, at some gather speed (the on-chip decode lengthens
 * each position's chain of dependent loads): 8 bytes are the faster width
 * for every form. Values are identical either way. Updates plan_bytes. No
 * counterpart in the reference. */
int emg_plan_set_record_width(emg_plan *plan, int bytes);

/* Host-only, between emg_plan_init and emg_plan_build: the element-value
 * layout of emg_assemble and of the plan's gather lists. EMG_LAYOUT_PACKED
 * (default): the canonical upper triangle, one record per (row, column pair)
 * contribution (record_bytes wide). EMG_LAYOUT_BLOCK: entity-pair blocks, one
 * 4-byte record per (row pair, column pair) contribution -- the two rows and
 * two columns of an entity pair come from the same tets, so one record and
 * one contiguous read give four entries of A. A is bit for bit the same in
 * both layouts. Updates plan_bytes. No counterpart in the reference. */
int emg_plan_set_value_layout(emg_plan *plan, int layout);

/* Builds the entity->tet incidence lists, column lengths and indptr[N+1]
 * (int32) on the device, then synchronises `stream` and stores nnz/max_col in
 * *plan. Replaces precompute_csc_pattern phases 1-3 (csc_cast.py:65-126) for
 * the structured Nedelec-2 pattern (rows of column c = DoFs of every entity
 * sharing a tet with c's entity). d_tets: int32[4][n_tets] (vertex ranks of
 * each tet go into the plan); d_tetids: int32[n_assy] or NULL (all tets). */
int emg_plan_build(emg_plan *plan, const int32_t *d_tets, const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri,
                   const int32_t *d_tetids, void *d_plan, void *d_workspace, int32_t *d_indptr, int64_t *d_status,
                   emg_stream_t stream);

/* Writes indices[nnz] (int32, sorted within each column), the per-slot column
 * positions and the gather lists (for each output position, its contributing
 * element slots in a fixed order). Replaces precompute_csc_pattern phase 4
 * (csc_cast.py:131-160). */
int emg_plan_finish(const emg_plan *plan, const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri,
                    const int32_t *d_tetids, void *d_plan, const int32_t *d_indptr, int32_t *d_indices,
                    int64_t *d_status, emg_stream_t stream);

/* Optional, after emg_plan_finish: orders the gather's entity chunks along a
 * Morton curve of their position (the centroid of each chunk's first incident
 * tet, quantised to 1024 cells per axis of the mesh's bounding cube), so that
 * chunks that share tets are gathered close together in time and the shared
 * element values are still in L2. Changes which warp computes which column
 * run and when, never a value. Without it the gather walks edge and face
 * chunks in a proportional interleave of their index order. d_workspace:
 * plan->workspace_bytes. No counterpart in the reference (a GPU memory
 * hierarchy optimisation). */
int emg_plan_order(const emg_plan *plan, void *d_plan, const double *d_nodes, int64_t n_nodes, const int32_t *d_tets,
                   const int32_t *d_tetids, void *d_workspace, emg_stream_t stream);

/* Element kernel: per assembled tet ia the 20x20 element block in `layout`
 * (EMG_LAYOUT_COO is the reference's dataE/dataB layout, 400 values per tet;
 * EMG_LAYOUT_PACKED 210). out = EMG_OUT_K gives the reference's dataE,
 * EMG_OUT_M its dataB, EMG_OUT_LINCOMB alpha*K_e + beta*M_e. d_values is
 * complex64 for EMG_MIXED and complex128 otherwise. Replaces
 * _matrix_builder (curlcurl.py:387-456) + ned2_tet_stiff_mass (:285-380). */
int emg_element_values(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                       const int32_t *d_tetids, int64_t n_assy, const emg_material *mat, int precision, int out,
                       int layout, double alpha_re, double alpha_im, double beta_re, double beta_im,
                       void *d_values, int64_t *d_status, emg_stream_t stream);

/* Column gather + segmented sum: A[nnz] (complex128, CSC order of the plan)
 * = sum over element slots of alpha*V1 + beta*V2, where V1 (required) and V2
 * (optional, NULL) are element-value arrays written by emg_element_values with
 * the same precision (complex64 for EMG_MIXED, complex128 otherwise) and
 * layout (EMG_LAYOUT_PACKED: V2 must be NULL). Deterministic (fixed summation order), no atomics.
 * Replaces CSCMapping.to_csc / scatter_to_csc_c16 (csc_cast.py:55-63, 162-177). */
int emg_gather(const emg_plan *plan, const void *d_plan, const int32_t *d_indptr, const void *d_v1,
               const void *d_v2, int precision, int layout, double alpha_re, double alpha_im, double beta_re,
               double beta_im, void *d_A, int64_t *d_status, emg_stream_t stream);

/* Bytes of element-value scratch that emg_assemble needs. */
size_t emg_assemble_workspace_size(int64_t n_assy, int precision);

/* One-call assembly of A = alpha*K + beta*M values in CSC order: element
 * kernel into d_workspace (emg_assemble_workspace_size bytes) + gather.
 * Replaces tet_mass_stiffness_matrices + to_csc(Evec - Bvec*k0^2)
 * (curlcurl.py:222-270 with a cached cscmap; assembler.py:485-494). */
int emg_assemble(const emg_plan *plan, const void *d_plan, const int32_t *d_indptr, const double *d_nodes,
                 int64_t n_nodes, const int32_t *d_tets, const int32_t *d_tetids, const emg_material *mat,
                 int precision, double alpha_re, double alpha_im, double beta_re, double beta_im, void *d_workspace,
                 size_t workspace_bytes, void *d_A, int64_t *d_status, emg_stream_t stream);

/* One job of emg_assemble_batch: the arguments of emg_assemble for one mesh.
 * d_values: that job's element-value workspace (emg_assemble_workspace_size
 * bytes for its n_assy), d_A: its nnz complex128 values; d_status may be
 * shared between jobs or NULL. */
typedef struct {
  const emg_plan *plan; /* host struct, read during the call */
  const void *d_plan;
  const int32_t *d_indptr;
  const double *d_nodes;
  int64_t n_nodes;
  const int32_t *d_tets;
  const int32_t *d_tetids;
  emg_material mat;
  double alpha_re, alpha_im, beta_re, beta_im;
  void *d_values;
  void *d_A;
  int64_t *d_status;
} emg_assembly_job;

/* Bytes of the job table of emg_assemble_batch for n_jobs jobs (the same
 * size on the host and on the device). */
size_t emg_assemble_batch_table_bytes(int n_jobs);

/* emg_assemble for n_jobs independent jobs in two launches: one element
 * kernel over all the jobs' tets, then one gather over all their entity
 * chunks (each CTA looks its job up in the table). Every job's A is bit for
 * bit what emg_assemble gives it alone. All jobs share one material kind,
 * the precision and the value layout (block plans, or packed ones with
 * 8-byte gather records). The table is written to h_table (host, emg_assemble_batch_table_bytes) and copied to
 * d_table on the stream: when h_table is page-locked the copy is
 * asynchronous and h_table must stay untouched until the stream has passed
 * this call. No counterpart in the reference (batching of independent
 * assembly jobs, a serving optimisation: a serving loop assembles K and M of
 * every job admitted since its last launch together). */
int emg_assemble_batch(const emg_assembly_job *h_jobs, int n_jobs, int precision, void *h_table, void *d_table,
                       size_t table_bytes, emg_stream_t stream);

/* emg_assemble without a workspace argument, for callers that cannot
 * allocate device memory at the call site (a plugin inside another
 * framework's pre-reserved device pool; a latency-bound loop that must not
 * call cudaMalloc/cudaFree, which synchronise the device). It has no
 * counterpart in the reference. The element-value scratch is a file-scope
 * device array of 96 MiB that every GPU loading this library holds until
 * exit: at most 28,597 assembled tets in EMG_FP64/EMG_EXACT, 57,195 in
 * EMG_MIXED; larger plans return EMG_ERANGE. It calls no cudaMalloc/cudaFree.
 * Every call looks the array's address up in the current device's context
 * (cudaGetSymbolAddress), so a device reset between calls is safe; the
 * first call on a device loads the module there, so make that first call
 * before any stream capture.
 * All calls share the array: calls that overlap on the GPU (other streams or
 * threads) race and corrupt each other's results. Inputs and outputs are the
 * caller's, as for emg_assemble. */
int emg_assemble_noalloc(const emg_plan *plan, const void *d_plan, const int32_t *d_indptr, const double *d_nodes,
                         int64_t n_nodes, const int32_t *d_tets, const int32_t *d_tetids, const emg_material *mat,
                         int precision, double alpha_re, double alpha_im, double beta_re, double beta_im, void *d_A,
                         int64_t *d_status, emg_stream_t stream);

/* A_f = a_f*K + b_f*M (+ c_f*P) for nf frequencies, complex128 CSC values of
 * one pattern: K, M (and P, may be NULL) read once per call. h_coef holds
 * nf*6 doubles (a_re, a_im, b_re, b_im, c_re, c_im) per frequency; d_out
 * points to nf arrays of nnz complex128, d_out[f] = base + f*out_stride
 * elements. Replaces the per-frequency to_csc(Evec - Bvec*k0^2) of the cached
 * sweep (assembler.py:472-494). */
int emg_form_sweep(const void *d_K, const void *d_M, const void *d_P, int64_t nnz, const double *h_coef, int nf,
                   void *d_out, int64_t out_stride, emg_stream_t stream);

/* One work item of the serving batch: out[i] = a*K[i] + b*M[i] + c*P[i] for
 * i < nnz (complex128; P may be NULL), coef = (a_re, a_im, b_re, b_im, c_re,
 * c_im). group: on the first of g consecutive items that share K, M, P and
 * nnz (one job's frequencies), g -- they are formed together, K, M and P read
 * once -- and 0 on the other g - 1; 1 for an item alone. The tile offsets
 * give the group's tiles to its first item and none to the others. 88 bytes. */
typedef struct {
  const void *K, *M, *P;
  void *out;
  int64_t nnz;
  int32_t group;
  int32_t reserved;
  double coef[6];
} emg_form_item;

/* Form of a batch of (job, frequency) items that may belong to different
 * meshes in one launch: the items are split into tiles of 32768 nonzeros and
 * a fixed grid of (SM count x 16) CTAs walks all tiles, a few per CTA. The item count and the
 * tile offsets are read from DEVICE memory (*d_n_items, d_tile_start[n+1]),
 * so one captured CUDA graph (a host-to-device copy of a new batch followed
 * by this launch) can be replayed for every batch. Serving-engine entry
 * point; its per-item arithmetic is the cached sweep's to_csc(Evec - Bvec*k0**2)
 * (assembler.py:472-494). */
int emg_form_batch(const emg_form_item *d_items, const int64_t *d_tile_start, const int32_t *d_n_items, int max_items,
                   emg_stream_t stream);

/* Robin (third-kind) boundary term of ports, absorbing boundaries and
 * surface impedances on boundary triangles. Replaces assemble_robin_bc /
 * compute_bc_entries / ned2_tri_stiff (physics/microwave/assembly/
 * robinbc.py:316-451) and the caller's K += field.generate_csc(B_robin)
 * (assembler.py:576-630). The triangle block is linear in gamma, so it is
 * built once (gamma = 1) and each frequency adds gamma(f) times it into A. */
typedef struct {
  int64_t n_btris;     /* boundary triangles (a triangle listed twice counts twice) */
  int64_t n_slots;     /* 64 per triangle: its 8x8 block */
  int64_t n_keys;      /* power of two >= n_slots: length of the sorted key array */
  size_t keys_bytes;   /* 8 * n_keys: d_keys of build/apply */
  size_t values_bytes; /* 16 * n_slots: d_values (complex128) of build/apply */
  int64_t n_fslots;    /* 8 per triangle: its forcing-vector entries */
  int64_t n_fkeys;     /* power of two >= n_fslots */
  size_t fkeys_bytes;  /* 8 * n_fkeys: d_fkeys of emg_robin_force */
  size_t fvalues_bytes; /* 16 * n_fslots: d_fvalues of emg_robin_force */
} emg_robin;

/* Host-only: sizes for n_btris triangles (fewer than 2^26). */
int emg_robin_init(int64_t n_btris, emg_robin *robin);

/* Per boundary triangle d_btris[i] (int32 index into tris): its 8x8 block for
 * gamma = 1 (6-point rule in the triangle's plane, robinbc.py:189-196) and the
 * position in A (the CSC pattern d_indptr/d_indices of N columns) of each of
 * its 64 (row, column) DoF pairs; keys sorted by position, then slot, so that
 * emg_robin_apply sums each position in a fixed order. d_tris, d_tri_to_edge:
 * int32 [3][n_tris] (sorted vertex ids; edges (v0,v1), (v1,v2), (v0,v2),
 * mesh3d.py:836-839). A pair outside the pattern (a triangle whose tets are
 * all excluded) sets EMG_ST_INDEX in d_status and is dropped. */
int emg_robin_build(const emg_robin *robin, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                    const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                    const int32_t *d_indptr, const int32_t *d_indices, int64_t N, uint64_t *d_keys, void *d_values,
                    int64_t *d_status, emg_stream_t stream);

/* emg_robin_build with the caller's DoF numbering: d_tri_dofs (int32
 * [n_btris][8]) gives each listed triangle's 8 DoFs in tri_to_field slot
 * order (3 ne0 edges, 3 ne2 edges, nf0, nf1). For the opposite side of a
 * ThinConductor these are the columns of tri_to_field_os (nedelec2.py:
 * 156-158), and the term is field.generate_csc(B2, empty_tri_rowcol(
 * other_side=True)) of assembler.py:605-608,636-639 (femdata.py:86-104): the
 * same blocks on the split DoFs. d_indptr/d_indices must already hold every
 * pair (the union pattern of emg_csc_lookup / emg_csc_shift). */
int emg_robin_build_dofs(const emg_robin *robin, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                         const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                         const int32_t *d_tri_dofs, const int32_t *d_indptr, const int32_t *d_indices, int64_t N,
                         uint64_t *d_keys, void *d_values, int64_t *d_status, emg_stream_t stream);

/* Pattern lookup: d_out[i] = the position of (d_rows[i], d_cols[i]) (int64)
 * in the CSC pattern d_indptr/d_indices of N columns, or -(1 + p) with p the
 * position the row would be inserted at in its column (INT64_MIN for an
 * index outside [0, N)). Used to lay out the union of A's pattern and extra
 * entries (scipy's csc + csc, which the reference's K += generate_csc(...)
 * performs, assembler.py:636-639). */
int emg_csc_lookup(const int32_t *d_indptr, const int32_t *d_indices, int64_t N, const int64_t *d_cols,
                   const int64_t *d_rows, int64_t n, int64_t *d_out, emg_stream_t stream);

/* Shifted copy into a grown pattern: d_dst[p + d_seg_shift[s]] = d_src[p] for
 * p < n_src, s the last segment with d_seg_start[s] <= p (d_seg_start[0] = 0,
 * ascending, n_seg entries), then d_dst[d_xpos[e]] = d_xval[e] (zero when
 * d_xval is NULL) for e < n_x. elem_bytes 16 (complex128 values), 8
 * (complex64) or 4 (int32 row indices). Positions outside [0, n_dst) are
 * skipped. One launch; HBM-bound. */
int emg_csc_shift(const void *d_src, int64_t n_src, int elem_bytes, const int64_t *d_seg_start,
                  const int64_t *d_seg_shift, int n_seg, const int64_t *d_xpos, const void *d_xval, int64_t n_x,
                  void *d_dst, int64_t n_dst, emg_stream_t stream);

/* The second-order absorbing boundary correction in place of the Robin
 * block, same descriptor, buffers, keys and emg_robin_apply: per triangle
 * B[a][b] = A sum_q w_q c_a c_b with c the scalar 2-D curls of the 8
 * functions (abc_order_2_matrix / _abc_order_2_terms,
 * physics/microwave/assembly/robin_abc_order2.py:143-281, with its own
 * 14-digit copy of the 6-point rule); apply it with the coefficient the
 * assembler passes (assembler.py:626-632: c2 = bc.get_abccorr(k0)). */
int emg_abc2_build(const emg_robin *robin, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                   const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                   const int32_t *d_indptr, const int32_t *d_indices, int64_t N, uint64_t *d_keys, void *d_values,
                   int64_t *d_status, emg_stream_t stream);

/* d_A[p] += gamma * (sum of the triangle slots at position p) for the nnz
 * values of A (complex128); stream-ordered, deterministic. */
int emg_robin_apply(const emg_robin *robin, const uint64_t *d_keys, const void *d_values, double gamma_re,
                    double gamma_im, void *d_A, int64_t nnz, emg_stream_t stream);

/* Port forcing vector: d_b[N] (complex128) += the boundary triangles'
 * ned2_tri_force entries (robinbc.py:220-313, assemble_robin_bc_bvec
 * :405-433) for the incident field d_U (complex128 [3][6][n_btris]: component,
 * quadrature point of the 6-point rule, triangle; the points are those of
 * generate_points_3d :104-135). Each DoF sums its triangles in list order.
 * Scratch d_fkeys / d_fvalues: robin->fkeys_bytes / fvalues_bytes. */
int emg_robin_force(const emg_robin *robin, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                    const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                    const void *d_U, uint64_t *d_fkeys, void *d_fvalues, void *d_b, int64_t N, int64_t *d_status,
                    emg_stream_t stream);

/* Solve-DoF submatrix: Asel = A[:, solve_ids][solve_ids, :] on the device
 * (solver.py:2071; solve_ids = the DoFs that are not PEC, assembler.py:
 * 543-564,742). d_keep: uint8 [N], 1 for a solve DoF. The pattern (indptr_sel
 * [M+1], indices_sel [nnz_sel], rows renumbered and ascending as scipy's
 * slicing gives them) and the take map (position in A of each selected
 * entry) are built once; emg_select_values gathers the values per frequency. */
typedef struct {
  int64_t N;              /* columns of A */
  int64_t M;              /* solve DoFs (set by emg_select_build) */
  int64_t nnz_sel;        /* nonzeros of Asel (set by emg_select_build) */
  size_t workspace_bytes; /* scratch of build and finish (keep it between them) */
} emg_select;

int emg_select_init(int64_t N, emg_select *sel);
/* d_indptr_sel needs N + 1 entries (M + 1 are used); synchronises stream. */
int emg_select_build(emg_select *sel, const int32_t *d_indptr, const int32_t *d_indices, const uint8_t *d_keep,
                     void *d_workspace, int32_t *d_indptr_sel, int64_t *d_status, emg_stream_t stream);
int emg_select_finish(const emg_select *sel, const int32_t *d_indptr, const int32_t *d_indices, const uint8_t *d_keep,
                      void *d_workspace, const int32_t *d_indptr_sel, int32_t *d_indices_sel, int32_t *d_take,
                      emg_stream_t stream);
/* d_A_sel[q] = d_A[take[q]] (complex128), q < nnz_sel. */
int emg_select_values(const emg_select *sel, const int32_t *d_take, const void *d_A, int64_t nnz, void *d_A_sel,
                      emg_stream_t stream);

/* Post-processing. The solution d_x (complex128 [N]) at points d_points
 * (f64 [3][n_points]) inside the tets d_tet_of (int32 [n_points]; -1 or an
 * invalid tet gives NaN, as the reference does for points outside): d_E
 * complex128 [3][n_points]. Replaces ned2_tet_interp
 * (compiled/base/interp.py:286-387) for points whose tet is known. */
int emg_ned2_interp(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                    const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri, int64_t n_edges, int64_t n_tris,
                    const void *d_x, const double *d_points, int64_t n_points, const int32_t *d_tet_of, void *d_E,
                    emg_stream_t stream);

/* Port overlap of the S-parameters: per port triangle d_btris[i] (lying on a
 * face of tet d_btets[i]) area * sum_k w_k (E - q U) . conj(U) at the points
 * of the triangle rule h_rule (host f64 [4][nq]: weights, L1, L2, L3; nq <=
 * 16), U complex128 [3][nq][n_btris]; d_per_tri complex128 [n_btris] and
 * *d_total their sum (fixed order). The integral of sparam_field_power
 * (physics/microwave/sparam.py:62-97, mth/integrals.py:64-103) times 2 Z0. */
int emg_port_overlap(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                     const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri, const int32_t *d_tris, int64_t n_edges,
                     int64_t n_tris, const void *d_x, const int32_t *d_btris, const int32_t *d_btets, int64_t n_btris,
                     const double *h_rule, int nq, const void *d_U, double q, void *d_per_tri, void *d_total,
                     int64_t *d_status, emg_stream_t stream);

/* Sparse direct solve of an n x n complex128 system on the device, the
 * handoff after emg_select_*: A x = b with A in CSR (0-based, int32). The
 * reference hands A[:, solve_ids][solve_ids, :] to SuperLU / Pardiso / MUMPS or
 * to cuDSS (SolverCuDSS, solver.py:1274-1323; slicing :2071); cuDSS is not in
 * this toolkit, so this calls cuSOLVER's sparse QR (cusolverSpZcsrlsvqr),
 * loaded on first use (EMG_EDEVICE if it cannot be). The CSC arrays of a
 * symmetric matrix (A = A^T, as every system this library assembles) are its
 * CSR arrays. tol: singularity threshold; reorder: 0 none, 1 symrcm, 2 symamd,
 * 3 metis (passed through). *h_singularity = -1 if A is invertible, else the
 * first row found dependent. Blocking; cuSOLVER allocates its own scratch. */
int emg_sparse_solve(int64_t n, int64_t nnz, const int32_t *d_row_ptr, const int32_t *d_col_ind, const void *d_values,
                     const void *d_b, void *d_x, double tol, int reorder, int64_t *h_singularity, emg_stream_t stream);

/* General COO -> CSC mapping: CSCMapping.from_rowcol / to_csc
 * (mth/csc_cast.py:51-177) for any slot list, as the heat-conduction assembly
 * uses it (physics/heatconduction/assembly/grad.py:403-460). Slots are
 * counted and scattered per column, each column's slots sorted by (row, slot)
 * (a fixed order), its distinct rows are its entries; an entry's value is the
 * sum of its slots in that order. Sizes from emg_coo_init: d_perm perm_bytes,
 * workspace workspace_bytes (keep it from build to finish), d_indptr N + 1;
 * then, with nnz set by emg_coo_build (which synchronises), d_indices nnz and
 * d_run nnz + 1 int32 (run_bytes bounds it before nnz is known). */
typedef struct {
  int64_t S, N, nnz;
  size_t perm_bytes, run_bytes, workspace_bytes;
} emg_coo_map;

int emg_coo_init(int64_t n_slots, int64_t N, emg_coo_map *map);
/* rows/cols of an element with D DoFs per tet: slot D^2 t + D ii + jj has row
 * t2f[ii] and column t2f[jj] (femdata.py:58-73); t2f int32 [D][n_tets]. */
int emg_coo_rowcol(const int32_t *d_tet_to_field, int dofs_per_tet, int64_t n_tets, int32_t *d_rows, int32_t *d_cols,
                   emg_stream_t stream);
int emg_coo_build(emg_coo_map *map, const int32_t *d_rows, const int32_t *d_cols, int32_t *d_perm, void *d_workspace,
                  int32_t *d_indptr, int64_t *d_status, emg_stream_t stream);
int emg_coo_finish(const emg_coo_map *map, const int32_t *d_rows, const int32_t *d_perm, void *d_workspace,
                   const int32_t *d_indptr, int32_t *d_indices, int32_t *d_run, emg_stream_t stream);
/* CSC values (f64, or complex128 when is_complex) from slot values:
 * block_dofs 0 reads slot s at d_values[s]; block_dofs 10 reads values stored
 * as transposed 10x10 blocks (EMG_LAYOUT_COO_T) of slots 100 t + 10 i + j. */
int emg_coo_gather(const emg_coo_map *map, const int32_t *d_perm, const int32_t *d_run, int is_complex, int block_dofs,
                   const void *d_values, void *d_out, emg_stream_t stream);

/* Heat conduction, Lagrange-2 (10 DoFs per tet): per tet the 10x10 block in
 * the reference's COO slots (row-major), kind 0 = stiffness with the
 * conductivity d_coef f64 [3][3][n_tets] (leg2_tet_stiff, grad.py:199-260),
 * kind 1 = mass with d_coef = rho_cp f64 [n_tets] (leg2_tet_mass :263-330).
 * precision EMG_FP64: the reference's quadrature loop and operation order;
 * EMG_EXACT: the same rule folded into per-tet moments (translation
 * invariant, no cancellation in the barycentrics). layout EMG_LAYOUT_COO (the
 * reference's row-major blocks) or EMG_LAYOUT_COO_T (transposed blocks). A
 * degenerate tet or bad node index sets d_status and gets a zero block. */
int emg_leg2_element(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                     const double *d_coef, int kind, int precision, int layout, double *d_values, int64_t *d_status,
                     emg_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* EMGPU_H */
