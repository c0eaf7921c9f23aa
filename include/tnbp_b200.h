/*
 * tnbp_b200 — C ABI of the B200 (sm_100a) loopy-BP PEPS expectation-value
 * engine.  Plain C: opaque handles, plain pointers and sizes, int status.
 *
 * Every entry point below replaces one function of r-ccs-cms/tnbp on the
 * estimator hot path; the replaced interface is cited as path:line within
 * that project.  The reference state is a set of caller-owned
 * std::vector<TenT> (site tensors V, messages E/F); here the same state lives
 * on the device inside a job handle and is mutated in place by these calls.
 *
 * Conventions shared with the reference (restated, not copied):
 *  - Sites are the sorted distinct labels of the edge list
 *    (GetSiteIndexFromBond, include/tnbp/framework/graph.h:23-35); a site is
 *    addressed here by its position in that sorted list ("site index").
 *  - Leg k of a site is the k-th edge, in edge-list order, that contains the
 *    site (GetSurroundingBondIndex, graph.h:40-55); the physical leg is last.
 *  - Tensors are column-major: coordinate 0 varies fastest.  Host buffers
 *    are interleaved complex128 (re, im) unless stated otherwise.
 *  - Messages: index m < n_edges is the message computed at edges[m].first
 *    (absorbed by .second); index m + n_edges is the one computed at
 *    edges[m].second (bp.h:170-174, 221-225).
 *  - Status: 0 = success; a negative TNBP_E* code on failure, with a
 *    readable message from tnbp_last_error() (per thread).  No call traps
 *    the GPU to report an error.
 */
#ifndef TNBP_B200_H
#define TNBP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define TNBP_OK 0
#define TNBP_EINVAL -1      /* bad argument (std::invalid_argument in the reference) */
#define TNBP_ECUDA -2       /* CUDA runtime error */
#define TNBP_ENOMEM -3      /* device allocation failed / over the HBM budget */
#define TNBP_ENOTCONV -4    /* bounded iteration limit reached (SVD sweeps) */
#define TNBP_EPARSE -5      /* QASM / Pauli text parse error (qasm::ParseError, runtime_error) */
#define TNBP_EUNSUPPORTED -6 /* gate or operator the reference also rejects */
#define TNBP_ENOGPU -7      /* no CUDA device visible */
#define TNBP_ECANCELED -8   /* the request was cancelled (tnbp_server_cancel) */

/* ---- precision of a job's device state ---- */
#define TNBP_C128 0 /* plain path: complex128 storage and arithmetic */
#define TNBP_C64 1  /* complex64 storage and BP sweeps (3xTF32 / FP32 products,
                       FP64 sums), FP64 truncation eigensolves */
#define TNBP_MIXED 2 /* mixed path: complex128 state (site tensors, messages),
                        BP sweeps on a complex64 copy of the site tensors
                        (3xTF32 / FP32 products, FP64 sums); AbsorbTPO,
                        truncation and measurement in FP64 */

typedef struct tnbp_job tnbp_job;
typedef struct tnbp_tpo tnbp_tpo;

/* Thread-local text of the last failure (empty string if none). */
const char* tnbp_last_error(void);
/* Library version string. */
const char* tnbp_version(void);
/* 1 if a CUDA device is visible, else 0.  Never fails. */
int tnbp_device_available(void);

/* ======================= host-side setup (bit-exact) ==================== */

/* bond_square_lattice (include/tnbp/lattice/square.h:14-34).
   Writes 2*(2*Lx*Ly-Lx-Ly) ints (pairs) to edges_out (capacity in pairs). */
int tnbp_square_lattice(int32_t Lx, int32_t Ly, int32_t* edges_out, int64_t cap_pairs,
                        int64_t* n_edges_out);

/* GreedyEdgeLayering (graph.h:138-170): layer_of_edge[i] = layer of edge i. */
int tnbp_greedy_layering(const int32_t* edges, int64_t n_edges, int32_t* layer_of_edge,
                         int32_t* n_layers_out);

/* GetSurroundingBondIndex (graph.h:40-55) for one site label. */
int tnbp_surrounding_bonds(const int32_t* edges, int64_t n_edges, int32_t site_label,
                           int32_t* bonds_out, int32_t cap, int32_t* n_out);

/* FindShortestPath (graph.h:57-108): BFS path src..dst (labels). */
int tnbp_shortest_path(const int32_t* edges, int64_t n_edges, int32_t src, int32_t dst,
                       int32_t* path_out, int32_t cap, int32_t* n_out);

/* qasm::parse_any (include/qasm/any.h:8-21) + EdgesFromQasm
   (include/tnbp/parser/qasmtoedge.h:38-56).  Writes sorted unique
   (min,max) pairs of the 2-qubit gates. */
int tnbp_qasm_edges(const char* qasm_src, int32_t* edges_out, int64_t cap_pairs,
                    int64_t* n_edges_out);

/* qasm::parse_any: flattened instruction list.  For instruction i:
   op[i] = qasm::Op enumerator value (include/qasm/ir.h:13-16),
   nq[i] qubit indices in qubits[4*i..], np[i] params in params[3*i..].
   Returns the count in n_out (call with cap 0 to size). */
int tnbp_qasm_instructions(const char* qasm_src, int32_t* op, int32_t* nq, int32_t* qubits,
                           int32_t* np, double* params, int64_t cap, int64_t* n_out);

/* pauli::load_sparse_pauli_op (include/pauli/sparse_pauli.h:52-97) on text,
   followed by SparsePauliToTensorOp + ClassifyOps
   (include/tnbp/parser/paulitotpo.h:39-153).  For each kept term t:
   kind[t] = 1 (one-site) or 2 (adjacent two-site); q0[t], q1[t] qubits
   (ascending); letters[2t], letters[2t+1] = 'X','Y','Z'; coeff[2t..2t+1]
   = (re, im); term_index[t] = its row in the file.  Terms the reference
   drops (identity, >2 qubits, non-adjacent pairs) are counted in
   n_dropped. */
int tnbp_pauli_terms(const char* text, const int32_t* edges, int64_t n_edges, int32_t* kind,
                     int32_t* q0, int32_t* q1, char* letters, double* coeff,
                     int32_t* term_index, int64_t cap, int64_t* n_kept, int64_t* n_dropped);

/* One TPO layer per barrier-delimited block of a QASM program
   (QasmToTPO, include/tnbp/parser/qasmtotpo.h:743-767, built with
   AppendGateToTPO 242-700 semantics).  Output for layer l:
   edge_rank[l*n_edges + e] = TPO bond dim on edge e; op data packed per
   site index in sorted-site order, each of shape (r_leg0..r_leg{g-1}, 2, 2)
   column-major, complex128 interleaved.  op_offset[l*n_sites+s] is the
   complex-element offset of site s in the packed buffer.  Call with
   cap_elems 0 to size (n_layers_out, total elements in n_elems_out). */
int tnbp_qasm_tpo(const char* qasm_src, const int32_t* edges, int64_t n_edges,
                  int32_t* edge_rank, int64_t* op_offset, double* op_data, int64_t cap_elems,
                  int32_t* n_layers_out, int64_t* n_elems_out);

/* QasmToTPO with manual gate-number layering (qasmtotpo.h:709-738, the
   estimator app's --num_gates): layer m takes the next num_gates[m]
   instructions; same output layout as tnbp_qasm_tpo.  A barrier, measure,
   reset or custom gate is TNBP_EUNSUPPORTED (the reference throws "matrix
   for this op not implemented"); more instructions than the counts cover,
   a layer that receives none, or a count < 1 is TNBP_EINVAL (undefined in
   the reference). */
int tnbp_qasm_tpo_counts(const char* qasm_src, const int32_t* edges, int64_t n_edges,
                         const int32_t* num_gates, int32_t n_counts, int32_t* edge_rank,
                         int64_t* op_offset, double* op_data, int64_t cap_elems,
                         int32_t* n_layers_out, int64_t* n_elems_out);

/* Kicked-Ising Floquet step as one TPO layer: exp(-i dt Jz ZZ) on every
   edge in edge order, then exp(-i dt hz Z), then exp(-i dt hx X) on every
   site (apps/kicked_ising_lattice/circuit.h:14-229).  The two-site gate is
   split with the operator-Schmidt rank it has (2, or 1 when sin or cos of
   dt*Jz vanishes); same output layout as tnbp_qasm_tpo with one layer. */
int tnbp_kicked_ising_tpo(const int32_t* edges, int64_t n_edges, double Jz, double hz,
                          double hx, double dt, int32_t* edge_rank, int64_t* op_offset,
                          double* op_data, int64_t cap_elems, int64_t* n_elems_out);

/* OptTPObySVD (include/tnbp/ptns/function/optsvdtpo.h:86-214) on one TPO
   layer, in place, as the reference mutates its std::vector<TenT>: for every
   edge in edge order the two site operators are contracted over their bond
   and split again by a truncated SVD that keeps the singular values > eps
   (at most the old bond dimension, at least one), sqrt(s) given to both
   sides.  On entry edge_rank[n_edges], op_offset[n_sites] (complex-element
   offsets relative to op_data) and op_data hold one layer in the layout of
   tnbp_qasm_tpo; on return they hold the compressed layer packed from
   op_data[0] in site order, n_elems_out its element count.  Bond dimensions
   never grow, so a layer packed without overlaps always fits.  Host code
   only (no device is used).  The reference app applies it to every layer
   after QasmToTPO when run with --do_opt_tpo (apps/estimator/main.cc:88-94). */
int tnbp_opt_tpo_svd(const int32_t* edges, int64_t n_edges, double eps, int32_t* edge_rank,
                     int64_t* op_offset, double* op_data, int64_t* n_elems_out);

/* ============================ device state =============================== */

/* InitTensorProductState (include/tnbp/ptns/function/init.h:18-95): product
   state |0...0> (site tensors of shape (1,...,1,d) holding e_0), every
   message the 1x1 tensor [1].  phys_dims may be NULL (all 2).  precision is
   TNBP_C128, TNBP_C64 or TNBP_MIXED.  stream is a cudaStream_t (NULL = a stream the job
   creates).  hbm_budget_bytes = 0 means no limit. */
int tnbp_job_create(const int32_t* edges, int64_t n_edges, const int32_t* phys_dims,
                    int32_t precision, void* stream, uint64_t hbm_budget_bytes, tnbp_job** out);
int tnbp_job_destroy(tnbp_job* job);
int tnbp_job_info(const tnbp_job* job, int64_t* n_sites, int64_t* n_edges, int32_t* precision);
/* Estimated peak device bytes of a job on this edge list whose BP runs at
   bond dimension bond_dim[e] on edge e (the largest it reaches; physical
   dimension 2): site tensors with their spare, chain and sweep-scratch
   buffers, message arenas, truncation work; the figure the server admits
   requests by.  Host only. */
int tnbp_footprint_estimate(const int32_t* edges, int64_t n_edges, const int32_t* bond_dim,
                            int32_t precision, uint64_t* bytes_out);
/* Bytes of device memory the job holds now. */
int tnbp_job_device_bytes(const tnbp_job* job, uint64_t* bytes);
/* Current bond dimension of every edge (n_edges ints). */
int tnbp_bond_dims(const tnbp_job* job, int32_t* dims_out);

/* Direct state access (the reference apps read/write std::vector<TenT>).
   Shapes follow the conventions above; rank = degree + 1. */
int tnbp_site_shape(const tnbp_job* job, int64_t site, int32_t* shape_out, int32_t cap,
                    int32_t* rank_out);
int tnbp_download_site(tnbp_job* job, int64_t site, double* data, int64_t cap_elems);
int tnbp_upload_site(tnbp_job* job, int64_t site, const int32_t* shape, int32_t rank,
                     const double* data);
int tnbp_download_message(tnbp_job* job, int64_t m, double* data, int64_t cap_elems,
                          int32_t* dim_out);
/* Sets message m (dim x dim).  Both messages of an edge must end with the
   edge's bond dimension before the next device call. */
int tnbp_upload_message(tnbp_job* job, int64_t m, int32_t dim, const double* data);

/* ============================== checkpoints ============================== */
/* Files in the layout of SaveTPS / LoadTPS
   (include/tnbp/ptns/function/iotps.h:37-105, apps/estimator_restart):
   size_t |V|, |Site_To_MpiRank|, |EdgeIdx|; the site tensors; SiteIdx; the
   (site, rank) pairs; the 2|EdgeIdx| messages; EdgeIdx.  Each tensor is
   uint64 order, int32 shape[order], complex128 scale (1), complex128 data
   column-major -- the record of gqten::tensor<std::complex<double>>::
   StreamWrite as restated for the reference's CPU build (gqten itself is not
   available).  These calls handle the whole state of one edge list held by
   one rank (every site on rank 0, EdgeIdx = 0 .. n_edges-1); a file written
   by one rank of several is rejected (TNBP_EINVAL). */

/* SaveTPS from host arrays: site tensors packed in sorted-site order, each of
   shape (bond_dim of its legs in leg order..., phys), then the 2*n_edges
   messages packed in order, message m of shape (bond_dim[m % n_edges])^2;
   complex128 interleaved.  phys_dims may be NULL (all 2). */
int tnbp_tps_write(const char* path, const int32_t* edges, int64_t n_edges, const int32_t* bond_dim,
                   const int32_t* phys_dims, const double* site_data, const double* msg_data);
/* LoadTPS into host arrays in the layout of tnbp_tps_write, after checking
   that the file holds the whole state of `edges` (site labels, edge ids,
   orders, shapes that agree on every bond).  Any output may be NULL;
   site_elems_out / msg_elems_out give the complex element counts. */
int tnbp_tps_read(const char* path, const int32_t* edges, int64_t n_edges, int32_t* bond_dim,
                  int32_t* phys_dims, double* site_data, int64_t site_cap, double* msg_data,
                  int64_t msg_cap, int64_t* site_elems_out, int64_t* msg_elems_out);
/* SaveTPS of a job's current site tensors and messages (the restart app's
   save after its last step, apps/estimator_restart/main.cc:253-257).  The
   file holds complex128 whatever the job's precision. */
int tnbp_save_state(tnbp_job* job, const char* path);
/* LoadTPS into a job created on the same edge list and physical dimensions
   (apps/estimator_restart/main.cc:84-92): bond dimensions, site tensors and
   messages are replaced.  A file that does not match leaves the job as it
   was; if device memory runs out after the check, destroy the job. */
int tnbp_load_state(tnbp_job* job, const char* path);

/* A TPO layer resident on the device (layout of tnbp_qasm_tpo, one layer). */
int tnbp_tpo_create(tnbp_job* job, const int32_t* edge_rank, const int64_t* op_offset,
                    const double* op_data, tnbp_tpo** out);
int tnbp_tpo_destroy(tnbp_tpo* tpo);

/* AbsorbTPO (include/tnbp/ptns/function/apply.h:15-177):
   V'[(v_k,o_k)..., p'] = sum_p O[o..., p, p'] V[v..., p] with merged bond
   index v + D*o, and every message E' = E (x) I_r. */
int tnbp_absorb_tpo(tnbp_job* job, const tnbp_tpo* tpo);

/* BeliefPropagation over all layers (bp.h:66-261) followed by the app's
   F -> E copy (apps/estimator/main.cc:140-143): one Jacobi sweep. */
int tnbp_bp_sweep(tnbp_job* job);

/* BeliefPropagationCondition (bp.h:266-355) of the current messages:
   mean over the 2|E| directed messages of
   || normalize(recomputed) - normalize(stored) ||_F. */
int tnbp_bp_condition(tnbp_job* job, double* result);

/* The apps' BP loop (apps/estimator/main.cc:131-157): up to max_iter sweeps,
   stop after the first whose condition is < tol.  Runs each sweep once
   (the condition of sweep k is the distance between sweep k+1 and sweep
   k, so the recomputation is shared).  iters_out = sweeps applied;
   cond_out = last condition (NaN if max_iter == 0).  On a TNBP_C64 or
   TNBP_MIXED job the
   tolerance used is max(tol, 1e-7) and, once the previous condition is
   below 1e-5, the loop also stops at the first sweep whose condition is
   larger than the previous one (keeping the messages before it): the
   complex64 condition has a rounding floor near 1e-7, and sweeping past
   the minimum only feeds unstable BP modes.  A non-finite condition fails
   with TNBP_ENOTCONV. */
int tnbp_bp_run(tnbp_job* job, double tol, int32_t max_iter, int32_t* iters_out,
                double* cond_out);

/* Truncation (include/tnbp/ptns/function/truncation.h:18-222 with
   SquareRootAndInverse, include/tnbp/framework/root.h:66-148): every edge
   in parallel, FP64 on the device.  bond_dims_out / trunc_err_out hold
   n_edges entries (may be NULL).  Rule for the kept singular values of
   T = Ra^T Rb / ||.||: s_i > sv_min, at most chi_max, at least one;
   trunc_err = discarded s^2 / total s^2. */
int tnbp_truncate(tnbp_job* job, int32_t chi_max, double sv_min, int32_t* bond_dims_out,
                  double* trunc_err_out);

/* Measure, one-site (include/tnbp/ptns/function/measure.h:15-94):
   out[2i..2i+1] = <O_i> at site index sites[i]; ops holds n 2x2 column-major
   operators (ops[8i..8i+7]) in the reference's O[p, p'] layout. */
int tnbp_measure_1site(tnbp_job* job, int64_t n, const int64_t* sites, const double* ops,
                       double* out);

/* Measure, nearest-neighbour two-site (measure.h:100-300): pairs[2i],
   pairs[2i+1] are site LABELS (a, b) of an edge; ops holds n (2,2,2,2)
   tensors O[p_a, p_b, p_a', p_b'] (ops[32i..32i+31]). */
int tnbp_measure_2site(tnbp_job* job, int64_t n, const int32_t* pairs, const double* ops,
                       double* out);

/* Sum_k c_k <P_k> in FP64 on the device over kept Pauli terms
   (same layout as tnbp_pauli_terms).  Not in the reference (which prints
   per-term values, apps/estimator/main.cc:213-238); per-term values are
   written to per_term_out (2 doubles each, may be NULL). */
int tnbp_measure_pauli_sum(tnbp_job* job, int64_t n_terms, const int32_t* kind,
                           const int32_t* q0, const int32_t* q1, const char* letters,
                           const double* coeff, double* per_term_out, double* sum_out);

/* Pauli products on any distinct qubits, including those ClassifyOps drops
   (include/tnbp/parser/paulitotpo.h:111-132: non-adjacent pairs, three or
   more qubits), which the reference does not measure.  Each term is
   measured on a tree cluster: the union of the shortest paths
   (FindShortestPath, graph.h:57-108) from its lowest-numbered qubit to the
   others (independent of the order the qubits are listed in),
   contracted exactly with its ket and bra layers, the Pauli letters on the
   qubit sites and the BP messages on every leg leaving the tree;
   <P> = Z(P) / Z(identity).  Exact where the graph is a tree (BP messages are
   exact environments there); for an adjacent pair it equals the two-site
   measurement.  n_qubits[t] >= 2; qubits and letters hold the terms one
   after another; values_out (2 doubles per term) and sum_out may be NULL. */
int tnbp_measure_cluster(tnbp_job* job, int64_t n_terms, const int32_t* n_qubits,
                         const int32_t* qubits, const char* letters, const double* coeff,
                         double* values_out, double* sum_out);

/* Every row of a sparse-Pauli text (load_sparse_pauli_op,
   include/pauli/sparse_pauli.h:52-97): kinds_out[row] = 0 identity, 1 one
   qubit, 2 adjacent pair (the two kinds ClassifyOps keeps; measured as
   tnbp_measure_pauli_sum does), 3 any other product.  With clusters == 0,
   kind-3 rows are not measured (NaN), as the reference drops them, and
   sum_out = sum over kinds 1 and 2; with clusters != 0 they are measured by
   tnbp_measure_cluster and sum_out adds them and the identity rows (value 1).
   values_out: 2 doubles per row.  Call with cap_rows 0 to size. */
int tnbp_measure_pauli_text(tnbp_job* job, const char* text, int32_t clusters, double* values_out,
                            int32_t* kinds_out, int64_t cap_rows, int64_t* n_rows_out,
                            double* sum_out);

/* Time spent in the job's last bp sweep kernels (ms, CUDA events) and the
   algorithmic flops/bytes of one sweep at the current shapes. */
int tnbp_sweep_stats(const tnbp_job* job, double* last_sweep_ms, double* flops,
                     double* bytes);

/* Sweep time summed over every sweep whose condition was read back (the BP
   loop reads each), with the matching algorithmic flops and bytes. */
int tnbp_sweep_totals(const tnbp_job* job, double* total_ms, double* total_flops,
                      double* total_bytes, int64_t* n_sweeps);

/* Kernels this process has launched through the library so far (a graph
   launch counts its kernel nodes). */
unsigned long long tnbp_kernel_launches(void);

/* No counterpart in the reference.  One directed BP message (the arithmetic
   of bp.h:128-175 for one site and one target leg) with NO device
   allocation, for callers that may not call cudaMalloc: code running inside
   a framework that owns the whole device-memory budget (a pre-reserved arena
   or an allocator that accounts for every byte) and code on a
   stream-ordered pipeline that cannot take cudaMalloc's implicit device
   synchronization.  Its scratch is one static device array of about 36 MiB
   that every GPU loading the library holds until exit; the caller passes
   device pointers to the inputs and the output:
     site      complex128 site tensor, column-major, shape[rank] with the
               physical leg last (at most TNBP_NOALLOC_MAX_SITE_ELEMS
               elements, bond dims <= 128; larger inputs are rejected with
               TNBP_EINVAL before any GPU work)
     msgs_in   host array of rank-1 device pointers: the incoming D_k x D_k
               message on each leg k (the entry for the target is ignored)
     msg_out   device pointer to D_t x D_t complex128: the normalized message
   The first call on a device looks up the scratch array's device address
   (cudaGetSymbolAddress) with that device current; make that first call
   before any stream capture.  Every call on a device shares the one array
   and overwrites it (nothing in it needs to start at zero), so calls whose
   GPU work overlaps race: order them on one stream or synchronize. */
#define TNBP_NOALLOC_MAX_SITE_ELEMS 1048576
int tnbp_bp_message_noalloc(const double* site, const int32_t* shape, int32_t rank,
                            int32_t target, const double* const* msgs_in, double* msg_out,
                            void* stream);

/* ============================ served path =============================== */

typedef struct tnbp_server tnbp_server;

/* Continuous-batching request loop on one GPU: jobs are admitted while
   their HBM footprint fits hbm_budget_bytes and max_active slots are free;
   BP sweeps of all active jobs run as one batched launch per stage. */
int tnbp_server_create(int32_t precision, uint64_t hbm_budget_bytes, int32_t max_active,
                       tnbp_server** out);
int tnbp_server_destroy(tnbp_server* srv);
/* Kicked-Ising estimator request on an L x L open square lattice:
   n_steps Floquet steps of RZZ(theta_j) on all edges then RX(theta_h) on all
   sites, BP(tol, max_iter), truncation to chi, then sum_k c_k <P_k>. */
int tnbp_server_submit_kicked_ising(tnbp_server* srv, int32_t L, int32_t chi, int32_t n_steps,
                                    double theta_j, double theta_h, double bp_tol,
                                    int32_t bp_max_iter, double sv_min, int64_t n_terms,
                                    const int32_t* kind, const int32_t* q0, const int32_t* q1,
                                    const char* letters, const double* coeff,
                                    int64_t* request_id);
/* Queue an estimator request for a QASM program and a sparse-Pauli
   observable (the estimator app's workload, apps/estimator/main.cc:105-238):
   edges = EdgesFromQasm, one TPO layer per barrier block (QasmToTPO), each
   compressed by OptTPObySVD when do_opt_tpo != 0; then per layer AbsorbTPO,
   the BP loop and Truncation to chi; finally the terms ClassifyOps keeps are
   measured and summed (Σ c_k <P_k>).  The TPO layers of a program are built
   and uploaded once and shared on the device by every request with the same
   program text and TPO options (least-recently-used cache of 32 programs;
   kicked-Ising requests are cached by (L, theta_j, theta_h) the same way).
   Parse errors return TNBP_EPARSE; a one-site term on a qubit that no
   two-qubit gate touches, TNBP_EINVAL. */
int tnbp_server_submit_qasm(tnbp_server* srv, const char* qasm_src, const char* pauli_text,
                            int32_t chi, double bp_tol, int32_t bp_max_iter, double sv_min,
                            int32_t do_opt_tpo, double eps_opt_tpo, int64_t* request_id);
/* TPO cache counters: look-ups served from the cache, layers built, and the
   programs held now. */
int tnbp_server_tpo_cache_stats(tnbp_server* srv, int64_t* hits_out, int64_t* misses_out,
                                int64_t* entries_out);
/* Cancel a request that has not finished: a queued one leaves the queue, an
   admitted one releases its device state and its share of the HBM budget at
   once (between server steps, so none of its work is in flight).  It is then
   done with TNBP_ECANCELED; cancelling a finished request is a no-op. */
int tnbp_server_cancel(tnbp_server* srv, int64_t request_id);
/* Advance the loop once (admission + one batched stage).  n_done_out =
   number of requests that completed during this call. */
int tnbp_server_step(tnbp_server* srv, int32_t* n_active_out, int32_t* n_queued_out,
                     int32_t* n_done_out);
/* Result of a finished request: sum (re, im); *pending_out = 0 if done, 1 if
   pending.  A request whose own work failed (non-finite BP condition,
   truncation error) is done and returns its error code (TNBP_ENOTCONV ...)
   with the message in tnbp_last_error(); the other requests are unaffected.
   A CUDA error fails tnbp_server_step itself. */
int tnbp_server_result(tnbp_server* srv, int64_t request_id, double* sum_out,
                       int32_t* pending_out);
/* Precision escalation (no counterpart in tnbp, whose estimator runs one
   precision): with on != 0, a TNBP_C64 or TNBP_MIXED server restarts, from
   |0...0> and in complex128, every request whose BP loop ends at its
   iteration limit without reaching its tolerance (the BeliefPropagation loop
   of apps/estimator/main.cc:131-157 running out of sweeps).  Non-converging
   BP is ill-conditioned: the messages after the last sweep carry every
   rounding of the earlier steps, amplified, so only the complex128 run
   reproduces the plain path's value.  Off by default; no effect on a
   TNBP_C128 server.  Requests already admitted keep running. */
int tnbp_server_set_escalation(tnbp_server* srv, int32_t on);
/* How a request ran: *precision_out = the precision of its last run,
   *escalated_out = 1 if it was restarted in complex128,
   *bp_converged_out = 1 if every BP loop of its last run reached its
   tolerance (0 if some loop stopped at the iteration limit).  Any pointer
   may be NULL; valid for queued, running and finished requests. */
int tnbp_server_request_info(tnbp_server* srv, int64_t request_id, int32_t* precision_out,
                             int32_t* escalated_out, int32_t* bp_converged_out);
/* Escalation threshold (no counterpart in tnbp): with escalation on, a
   request is restarted in complex128 only when the BP loop that ran out of
   sweeps never brought its condition (the mean message change per sweep,
   bp.h:266-355) below min_cond.  0 (the default) escalates on every loop
   that runs out of sweeps.  A loop whose condition came down to a small value
   and hovers there (a slow approach, a small limit cycle, the reduced
   precision's rounding floor) leaves messages that rounding moves little; a
   loop whose condition stays of order one is the ill-conditioned case.
   min_cond must be finite and >= 0 (TNBP_EINVAL otherwise). */
int tnbp_server_set_escalation_threshold(tnbp_server* srv, double min_cond);
/* BP statistics of a request's last run: *unconverged_loops_out = BP loops
   that stopped at the iteration limit, *worst_final_cond_out = the largest
   final condition among them, *worst_min_cond_out = the largest of their
   smallest conditions (0 when every loop converged).  Any pointer may be
   NULL. */
int tnbp_server_request_bp_stats(tnbp_server* srv, int64_t request_id, int32_t* unconverged_loops_out,
                                 double* worst_final_cond_out, double* worst_min_cond_out);

#ifdef __cplusplus
}
#endif

#endif
