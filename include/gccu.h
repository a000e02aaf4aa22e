/*
 * gccu.h -- C ABI of the B200 engine for GeCCo's blocked tensor contraction.
 *
 * Drop-in boundary: the Fortran host (formula interpreter frm_sched2, solvers)
 * stays unchanged and calls these entry points through ISO_C_BINDING from a
 * thin bind(C) shim module.  Conventions follow the reference:
 *   - every integer is int64_t (the reference is built with 64-bit default
 *     INTEGER, config/x86_64-linux.conf:39,51), reals are double;
 *   - irreps, occupation-class indices and Ms indices are 1-based;
 *   - an occupation is int64_t occ[2][4]: row 0 = creators, row 1 =
 *     annihilators, columns = hole, particle, valence, external (the
 *     reference's iocc(ngastp,2) transposed to C order);
 *   - every call returns 0 on success and a non-zero status on failure; the
 *     message is available from gccu_last_error (the shim turns a non-zero
 *     status into quit(1,...), baserout/quit.F).
 * Calls are not thread-safe (the reference host is single-threaded); all work
 * is ordered on one CUDA stream; calls that return numbers to the host
 * (norms, energies, downloads) synchronise that stream.
 */
#ifndef GCCU_H
#define GCCU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- life cycle ----------------------------------------------------------
 * replaces: memory set-up of gecco.x (gecco/gecco.f:125-130, mem_init);
 * memmax_bytes caps the device memory the engine may hold (<=0: no cap).
 * device < 0 starts a host-only engine: orbital model, graphs, ME-list
 * layouts and contraction plans can be queried, nothing is executed. */
int gccu_init(int64_t device, int64_t memmax_bytes);
int gccu_finalize(void);
/* device memory the engine holds (ME lists, maps, plans, workspaces) and its
 * cap (0: none), in bytes; replaces mem_free_words (memman/mem_free_words.f:2-9),
 * free = cap - used when a cap is set */
int gccu_mem_info(int64_t* used_bytes, int64_t* cap_bytes);
/* the device the engine runs on and the build of its kernels: info4 =
 * (compute capability 10*major+minor, SM count, binary and PTX version of
 * the tensor-core contraction kernel, 100 for sm_100a).  No counterpart in
 * the reference (a host query, like the banner of gecco/gecco.f). */
int gccu_device_info(int64_t* info4);
/* copies the last error message (NUL-terminated, truncated to len) */
int gccu_last_error(char* buf, int64_t len);

/* ---- orbital space ---------------------------------------------------------
 * replaces: orb_info set-up (include/def_orbinf.h; input/read_env_*.f).
 * norb_hpvx[t*8+g] = number of active (non-frozen, non-deleted) orbitals of
 * type t (0=H,1=P,2=V,3=X) in irrep g+1, g < nsym.  nsym in {1,2,4,8}. */
int gccu_register_orbinfo(int64_t nsym, const int64_t* norb_hpvx);

/* ---- graphs (string spaces) ------------------------------------------------
 * replaces: set_graph2 / weight_* (strings/set_graph2.f:2-206).
 * Number of strings of the graph (type,nel) with Ms index idxms (1..nel+1,
 * Ms = nel-2*(idxms-1)) and irrep gam. */
int gccu_graph_nstr(int64_t type, int64_t nel, int64_t idxms, int64_t gam, int64_t* nstr);
/* lexical address of one string (idx4sg, strings/idx4sg.f:2-82): orb[] 1-based
 * orbital numbers within the type, spn[] +1/-1/2 (2 = doubly occupied, listed
 * twice), in canonical order; returns the 0-based index within its block. */
int gccu_graph_index(int64_t type, int64_t nel, const int64_t* orb, const int64_t* spn,
                     int64_t* index);
/* the strings of one graph block in address order: n*nel entries of orb[]
 * (1-based) and spn[] (+1/-1/2); *n = number of strings (a host filling ME
 * lists uses these to place integrals, cf. input/import_h2_molpro_dump.f) */
int gccu_graph_strings(int64_t type, int64_t nel, int64_t idxms, int64_t gam, int64_t* orb,
                       int64_t* spn, int64_t maxn, int64_t* n);
/* one block of the signed string map, built on the device
 * (set_strmap_kernel, strings/set_strmap_kernel.f:66-119): entry
 * m[i2*n1+i1] = sign*(index12+1), 0 if Pauli-forbidden. */
int gccu_strmap_block(int64_t type, int64_t nel1, int64_t nel2, int64_t idxms1,
                      int64_t idxms2, int64_t gam1, int64_t gam2, int64_t* map, int64_t n);

/* ---- operators and ME lists -------------------------------------------------
 * replaces: operator definition (include/def_operator.h) + set_op_dim2
 * (operators/set_op_dim2.f:1-531).  occ: nblk occupation classes. */
int gccu_define_operator(const int64_t* occ, int64_t nblk, int64_t* op_id);
/* joined (multi-vertex) operator, op%njoined > 1 (include/def_operator.h):
 * occ holds nblk*njoined occupations, the njoined vertices of a class
 * consecutive (the reference's ihpvca_occ(ngastp,2,njoined*nblk)); ME lists
 * of it are laid out over the condensed components of all vertices
 * (operators/condense_occ.f, operators/set_op_dim2.f). Such lists can be
 * reordered, added and transferred; gccu_contract takes single-vertex
 * operands only in this engine version. */
int gccu_define_operator_joined(const int64_t* occ, int64_t njoined, int64_t nblk,
                                int64_t* op_id);
/* ME list of an operator with total irrep gamt, total 2*Ms mst and spin-flip
 * symmetry absym (0,+1,-1); its data live in device memory for the whole
 * solve (include/def_me_list.h:37-115).  Returns handle and len_op. */
int gccu_register_list(int64_t op_id, int64_t gamt, int64_t mst, int64_t absym,
                       int64_t* list_id, int64_t* len_op);
/* off_op_occ / len_op_occ of occupation class iblk (1-based) */
int gccu_list_block(int64_t list_id, int64_t iblk, int64_t* off, int64_t* len);
/* distribution table (same rows as the oracle): (iblk, idxmsa, gama, idxdis,
 * offset, length, ld, did); returns the row count in *nrows */
int gccu_list_dists(int64_t list_id, int64_t* rows, int64_t maxrows, int64_t* nrows);
/* host <-> device transfer of a whole list (replaces get_vec/put_vec,
 * fileutil/get_vec.f, for lists that are resident on the device) */
int gccu_upload_list(int64_t list_id, const double* host, int64_t n);
int gccu_download_list(int64_t list_id, double* host, int64_t n);
int gccu_zero_list(int64_t list_id);
/* ranged transfer of n elements starting at element offset (0-based):
 * replaces get_vec/put_vec (fileutil/get_vec.f, put_vec.f); src/dst may be
 * host (pageable or pinned) or device pointers */
int gccu_put_vec(int64_t list_id, int64_t offset, const void* src, int64_t n);
int gccu_get_vec(int64_t list_id, int64_t offset, void* dst, int64_t n);
/* raw device pointer of the list data (for callers that own device memory;
 * a frozen list must not be written through it) */
int gccu_list_device_ptr(int64_t list_id, void** dptr);
/* frozen != 0: the host declares the list's data constant until it is
 * unfrozen (the Hamiltonian lists during a CC solve, which the reference's
 * solver only reads, solve/solve_nleq.f).  Contractions planned while an
 * operand's list is frozen make the panels they derive from it (gathered
 * FP64 panels of map-addressed operands, split TF32 panels) once and keep
 * them; every entry point that would write a frozen list fails.  frozen = 0:
 * the cached panels are remade by the next contraction that reads them, and
 * CUDA graphs captured while they were valid can no longer be launched.  No
 * counterpart in the reference. */
int gccu_freeze_list(int64_t list_id, int64_t frozen);

/* ---- [CONTR] ------------------------------------------------------------------
 * replaces: contr_op1op2 case(2,3) (contract/contr_op1op2.f:112-173) ->
 * contr_op1op2_wmaps_c (contract/contr_op1op2_wmaps_c.f:2-2169) with the
 * inner kernels contr_blk1blk2_wmaps_c / contr_blk1blk2_blocked_mm.
 * Operands: occupation classes iblk_op1/iblk_op2 of lists list_op1/list_op2,
 * result class iblk_res of list_res.  occ_ex1/occ_ex2/occ_cnt are the
 * external / contracted parts (op1 = ex1+cnt, op2 = ex2+cnt^+,
 * res = ex1+ex2).  fact = bc_sign*contr%fac from the formula file
 * (formula/process_bc.f:528-535).  update=0 overwrites the result class.
 * use_tr: spin-flip symmetry (calculate.routes.use_tr), applied when all three
 * lists carry absym != 0.  type_xret: 0 none, 1 squared norm of the result
 * class, 2 its first element (scalars); written to *xret.
 * tra_op1/tra_op2/tra_res != 0: that class is used as its adjoint (the
 * vertex's dagger flag, contract/get_bc_info3.f:173,191,391); the occ_*
 * fields then describe the contraction of the adjoint, whose element
 * (C strings I, A strings J) is the stored element (C = J, A = I), total Ms
 * negated (contract/contr_op1op2_wmaps_c.f:427-429).  Operators of one
 * vertex only. */
typedef struct gccu_bc_desc {
  int64_t list_op1, iblk_op1;
  int64_t list_op2, iblk_op2;
  int64_t list_res, iblk_res;
  int64_t tra_op1, tra_op2, tra_res;
  int64_t occ_ex1[8], occ_ex2[8], occ_cnt[8];
} gccu_bc_desc;
int gccu_contract(const gccu_bc_desc* bc, double fact, int64_t update, int64_t use_tr,
                  int64_t type_xret, double* xret);
/* the block contractions the engine plans for a [CONTR] (without running
 * them): number of block contractions and the reference dgemm accounting of
 * gccu_stats for this contraction alone */
int gccu_plan_info(const gccu_bc_desc* bc, int64_t use_tr, int64_t* nitems, double* stats8);
/* the planned block contractions of a [CONTR] (planning only, also without a
 * device): up to maxrows rows of (M, N, K, map components of op1, of op2, of
 * the result, op1 contiguous along the contraction, op2 likewise); *nrows =
 * number of block contractions.  No counterpart in the reference (its
 * contr_op1op2_wmaps_c prints the same dimensions at ntest >= 100). */
int gccu_plan_items(const gccu_bc_desc* bc, int64_t use_tr, int64_t* rows8, int64_t maxrows,
                    int64_t* nrows);
/* [CONTR] without any device allocation.  No counterpart in the reference.
 * For callers that must not allocate device memory while they run: a host
 * that has given all device memory to its ME lists up front, or one that must
 * not stall the device, since cudaMalloc and cudaFree may synchronise it and
 * hold up work queued on other streams.  Same arguments and result as
 * gccu_contract with type_xret = 0, but the operand panels and the launch
 * descriptors go to one fixed device array compiled into the library
 * (64 MiB of panels, descriptors for 16384 block contractions) instead of
 * memory owned by the contraction; larger contractions are rejected with an
 * error naming the size they need.  The contraction must have been run once
 * through gccu_contract with the same descriptor and use_tr, because
 * planning allocates; the plan, including the operand panels planning
 * allocated for gccu_contract, stays allocated; this call allocates nothing
 * further.  The first call of an engine looks up the array's device address
 * (set-up, no allocation) and must come before any stream capture: inside
 * a capture it is rejected with an error.  Every call uses the same array
 * and leaves its contents behind; calls that overlap in time (from other
 * host threads or on other streams) race on it. */
int gccu_contract_noalloc(const gccu_bc_desc* bc, double fact, int64_t update, int64_t use_tr);

/* ---- [REORDER] ------------------------------------------------------------------
 * replaces: fs_reo_drv -> reo_op_wmaps_c -> reo_blk_wmaps_c
 * (contract/fs_reo_drv.f:166-173, contract/reo_op_wmaps_c.f,
 * contract/reo_blk_wmaps_c.f:2-854).  Occupation class iblk_ori of list_ori
 * is reordered into class iblk_reo of list_reo; both operators have the same
 * njoined.  Shift s (s < nshift <= 4), with occupation occ_shift[s] (layout as
 * in gccu_bc_desc), leaves vertex from_vtx[s] (1-based) of the original class
 * and arrives at vertex to_vtx[s] of the reordered one (the reference's
 * reorder occ_shift / from_vtx / to_vtx); all other strings keep their
 * vertex.  reo = (update ? reo : 0) + fac*sign_reo*(map signs)*ori, summed
 * over every way of splitting the merged strings; sign_reo is the formula's
 * reorder sign (contract/sign_reo.f, passed on by get_reo_info2.f:326).
 * type_xret as for gccu_contract, for the reordered class. */
typedef struct gccu_reo_desc {
  int64_t list_ori, iblk_ori;
  int64_t list_reo, iblk_reo;
  int64_t nshift;
  int64_t occ_shift[4][8];
  int64_t from_vtx[4], to_vtx[4];
} gccu_reo_desc;
int gccu_reorder(const gccu_reo_desc* reo, double fac, int64_t sign_reo, int64_t update,
                 int64_t type_xret, double* xret);
/* number of distribution cases and elements the engine plans for a reorder */
int gccu_reorder_info(const gccu_reo_desc* reo, int64_t* ncases, int64_t* nelements);

/* ---- self-contraction (partial trace) ----------------------------------------
 * replaces: contr_op1op2 -> trace_op -> trace_op_blk for a [CONTR] whose two
 * operands are the same operator (contract/contr_op1op2.f:162-169,
 * contract/trace_op.f:2-830, contract/trace_op_blk.f:2-178), without a
 * reordered result:
 *   res(IC,IA) = (update ? res : 0) + fact * sum_J op(IC*J, IA*J),
 * the contracted strings J identical on the creator and annihilator side
 * (occ_cnt: creator row equal to annihilator row).  fact = xfac*bc_sign as
 * for gccu_contract; type_xret as for gccu_contract.  Single-vertex
 * operators. */
int gccu_trace(int64_t list_op, int64_t iblk_op, int64_t list_res, int64_t iblk_res,
               const int64_t* occ_cnt, double fact, int64_t update, int64_t type_xret,
               double* xret);
/* number of distribution cases and elements the engine plans for a trace */
int gccu_trace_info(int64_t list_op, int64_t iblk_op, int64_t list_res, int64_t iblk_res,
                    const int64_t* occ_cnt, int64_t* ncases, int64_t* nelements);

/* ---- [ADD] -------------------------------------------------------------------
 * replaces: add_opblk (contract/add_opblk.f:2-313), in-core branch
 * :299-307: out(iblkout) = (reset ? 0 : out) + fac*in(iblkin); type 1 returns
 * the squared norm of the updated block, type 2 its first element. */
int gccu_add_block(double fac, int64_t list_in, int64_t iblk_in, int64_t list_out,
                   int64_t iblk_out, int64_t reset, int64_t type, double* xnorm2);
/* transposed [ADD] (fs_add_drv with tra_op != tra_res,
 * contract/fs_add_drv.f:127-131 -> add_opblk_transp,
 * contract/add_opblk_transp.f:2-355): out(IC,IA) = (reset ? 0 : out) +
 * fac*in(IA,IC), the input class being the adjoint of the output class
 * (total Ms negated, same IRREP); exactly one of tra_in, tra_out is set and
 * selects set_op_ldim_c's A-C sequence for that side; type as for
 * gccu_add_block.  Single-vertex operators. */
int gccu_add_block_transp(double fac, int64_t list_in, int64_t iblk_in, int64_t list_out,
                          int64_t iblk_out, int64_t tra_in, int64_t tra_out, int64_t reset,
                          int64_t type, double* xnorm2);
/* scale a whole list in place (scale_copy_op with one operand) */
int gccu_scale_list(int64_t list_id, double fac);
/* dot product of two lists of identical layout (DIIS subspace products) */
int gccu_dot_lists(int64_t list_a, int64_t list_b, double* dot);

/* ---- spin-flip symmetrisation ---------------------------------------------
 * replaces: sym_ab_blk (contract/sym_ab_blk.f:2-405) for one class:
 * x <- prefac*(x + relfac*flip(x)) */
int gccu_sym_ab(int64_t list_id, int64_t iblk, double prefac, double relfac);

/* ---- spin projection -----------------------------------------------------
 * replaces: spin_prj_list (contract/spin_prj_list.f:2-215) with
 * spin_prj_blk (contract/spin_prj_blk.f:2-527), the end-of-target step of
 * frm_sched2 for result lists with a spin (contract/frm_sched2.f:146-149):
 * every occupation class of the list is projected onto its singlet part in
 * place.  s2 (= 2S) must be 0 and the list's total Ms 0, as in the
 * reference; each class needs as many creators as annihilators (at most
 * four; a scalar class is left as it is).  xnorm2_blk (may be NULL): one
 * value per occupation class, the squared norm of the projected class
 * (spin_prj_list's update_norm); must be NULL inside a graph capture.  The
 * plan is made on the first call for a list (not inside a capture). */
int gccu_spin_prj_list(int64_t list_id, int64_t s2, double* xnorm2_blk);

/* ---- formula evaluation --------------------------------------------------
 * replaces: the command loop of frm_sched2 (contract/frm_sched2.f:117-365)
 * for one formula, with fs_newintm_drv / fs_delintm_drv (the [NEW] / [DEL]
 * intermediate commands, :239-252).  A formula is defined once
 * (gccu_formula_define) as an array of items and run any number of times
 * (gccu_formula_run), also inside a graph capture.  Intermediates are lists
 * registered with gccu_register_intermediate: they have no memory of their
 * own; when the formula is defined each gets a fixed byte range of one arena
 * owned by the formula, shared with the intermediates whose [NEW] .. [DEL]
 * windows do not overlap its own (first fit in the order of the [NEW]s), so
 * the arena holds the largest set of intermediates alive at one time instead
 * of all of them.  The addresses never change, so plans and captured graphs
 * stay valid.  An intermediate belongs to one formula and is named only
 * between its [NEW] and its [DEL] (or the end of the formula); outside a run
 * of that formula its contents are undefined. */
#define GCCU_CMD_TARGET 1  /* [INIT TARGET]: item.list becomes the target; init != 0 zeroes
                              it; mult = 2S+1 of the spin the list is projected onto at the
                              target's end (spin_prj_list for me_res%s2 = mult-1 >= 0,
                              frm_sched2.f:146-149): 1 = singlet, the only one; 0 = none */
#define GCCU_CMD_NEW 2     /* [NEW] intermediate item.list */
#define GCCU_CMD_DEL 3     /* [DEL] intermediate item.list */
#define GCCU_CMD_ADD 4     /* [ADD] (fs_add_drv): class iblk_out of item.list =
                              (reset ? 0 : itself) + fac * class iblk_in of list_in; with
                              tra_in or tra_out the transposed add (gccu_add_block_transp) */
#define GCCU_CMD_CONTR 5   /* [CONTR] (fs_contr_drv): gccu_contract(&bc, fac, update, use_tr) */
#define GCCU_CMD_REORDER 6 /* [REORDER] (fs_reo_drv): gccu_reorder(&reo, fac, sign_reo, update) */
typedef struct gccu_formula_item {
  int64_t command;
  int64_t list;
  int64_t init, mult;
  int64_t list_in, iblk_in, iblk_out, reset, tra_in, tra_out;
  int64_t update, use_tr, sign_reo;
  double fac;
  gccu_bc_desc bc;
  gccu_reo_desc reo;
} gccu_formula_item;
/* an ME list without memory of its own (an intermediate of a formula) */
int gccu_register_intermediate(int64_t op_id, int64_t gamt, int64_t mst, int64_t absym,
                               int64_t* list_id, int64_t* len_op);
int gccu_formula_define(const gccu_formula_item* items, int64_t n, int64_t* formula_id);
/* runs the items in order on the engine's stream.  xret (may be NULL: then
 * nothing is read back and the run may be captured in a graph): per
 * [INIT TARGET] item, in order, the target's value after its last item --
 * the element of a one-element list, else the list's 2-norm (frm_sched2's
 * xret); nxret must be at least the number of targets */
int gccu_formula_run(int64_t formula_id, double* xret, int64_t nxret);
/* info4: arena bytes, bytes of the intermediates one by one, targets, items */
int gccu_formula_info(int64_t formula_id, int64_t* info4);
/* byte offset of an intermediate in its formula's arena, -1 before its formula is defined */
int gccu_intermediate_offset(int64_t list_id, int64_t* offset);

/* ---- preconditioner ------------------------------------------------------
 * replaces: diavc (baserout/diavc.f:31-35) on whole lists:
 * out = fac*in/(diag+shift), |diag+shift| <= 1e-10 -> 1e-10 */
int gccu_precondition(int64_t list_out, int64_t list_in, int64_t list_diag, double fac,
                      double shift);

/* ---- learned correction of the preconditioner (no counterpart in the
 * reference, whose step is diavc, baserout/diavc.f:31-35, inside
 * optc_diis_sbsp_add, solve/optc_diis_sbsp_add.f:125-145) -------------------
 * A perceptron maps three inputs of every element to a factor m = 1 +
 * tanh(o) of the plain step s = fac*in/d, d = diag+shift clamped as in diavc:
 *   out = s * m,  inputs x0 = d/4, x1 = 1/max(|d|, 0.05),
 *   x2 = clip(u*v, -10, 10), u = s/rms(s), v = prev/rms(prev)
 * (prev = the previous step, list_prev; 0 = none, then v = 0);
 * h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), o = W3.h2 + b3, in FP64.
 * Weights: GCCU_LP_NWEIGHTS doubles, W1[32][3], b1[32], W2[32][32], b2[32],
 * W3[32], b3.  Training: sample rows (x0, x1, x2, s, amplitude) of chosen
 * elements during earlier solves (gccu_lp_rows), targets = converged
 * amplitude - sampled amplitude, loss L = mean over rows of
 * (s*(1+tanh(o)) - target)^2, gradients and Adam on the device. */
#define GCCU_LP_NWEIGHTS 1217
int gccu_lp_set_weights(const double* w, int64_t n);
int gccu_lp_get_weights(double* w, int64_t n);
int gccu_lp_precondition(int64_t list_out, int64_t list_in, int64_t list_diag,
                         int64_t list_prev, double fac, double shift);
/* rows[5*r..] = (x0, x1, x2, s, amplitude) of element idx[r] (0-based) of
 * lists in/diag/prev/amp (prev, amp: 0 = none) */
int gccu_lp_rows(int64_t list_in, int64_t list_diag, int64_t list_prev, int64_t list_amp,
                 double fac, double shift, const int64_t* idx, int64_t n, double* rows);
/* the training set: n rows of 5 (the fifth entry is not read) and targets */
int gccu_lp_load_samples(const double* rows, const double* target, int64_t n);
/* dL/dw over the whole training set (grad[GCCU_LP_NWEIGHTS]) and L */
int gccu_lp_gradient(double* grad, double* loss);
/* `steps` Adam steps (learning rate lr), each on `batch` rows drawn from the
 * set by a hash of (seed, step); *loss = the last minibatch's loss */
int gccu_lp_train(int64_t steps, int64_t batch, double lr, int64_t seed, double* loss);

/* ---- CUDA graphs -------------------------------------------------------------
 * Capture the device work of a sequence of calls (one formula evaluation,
 * contract/frm_sched.f:89-100) and replay it.  Calls inside a capture must not
 * request host values (type_xret must be 0); plans are cached per descriptor,
 * so a sequence is normally run once eagerly before it is captured. */
int gccu_graph_begin(void);
int gccu_graph_end(int64_t* graph_id);
int gccu_graph_launch(int64_t graph_id);
int gccu_sync(void);
/* Precision of the contractions planned after this call (no counterpart in
 * the reference, whose route-3 products are FP64 dgemm): 0 = FP64 on the FP64
 * tensor pipe (default); 1 = split TF32 on the tcgen05 tensor cores for the
 * GEMM-sized block contractions: each operand is split into two TF32 terms,
 * three products accumulate in FP32 over at most 4096 contraction indices,
 * and the partial results are added in FP64 (about FP32 accuracy per
 * product; items with at most 32 rows or columns or fewer than 256
 * contraction indices stay FP64); 2 = FP64 emulated on the int8 tensor
 * cores for the same block contractions: each operand row is cut into five
 * signed 8-bit slices under the row's scale (maximum / 127), the slice
 * products of order s + t < 5 are summed exactly in int32 and combined in
 * FP64 (about 35 bits of each operand relative to its row maximum); 3 = the
 * same with four slices (10 products, 28 bits, tiles up to 128 columns);
 * modes 2 and 3 are not supported by gccu_contract_noalloc.  Plans are kept
 * per mode, so a
 * solver can switch precision for its final iterations.  A pipeline wait
 * that times out inside a kernel is reported as an error by the next call
 * that synchronises (gccu_sync, norms, downloads). */
int gccu_set_precision(int64_t mode);
/* Owner-computes sharding of contractions over nranks devices (one engine
 * per rank, no counterpart in the reference): contractions run after this
 * call execute only this rank's share of their output tiles, the contiguous
 * range [n*rank/nranks, n*(rank+1)/nranks) of each tile list n (operand
 * gathers and splits run in full); the host sums the partial results of the
 * ranks (an all-reduce of the residual lists) and keeps everything else
 * replicated.  (0, 1) restores whole contractions.  Contractions planned
 * while nranks > 1 use the fixed tile rule even with gccu_set_tuning(1):
 * the shares partition the work only if every rank builds the same tile
 * lists. */
int gccu_set_shard(int64_t rank, int64_t nranks);
/* Polls of one pipeline wait of the tensor-core kernel before it gives up
 * (polls < 0: the default, 4194304); on time-out the kernel stops, waits for
 * the work it has issued, sets the engine's error flag and returns, and the
 * next synchronising call reports the error.  No counterpart in the
 * reference (failure detection of the device pipeline). */
int gccu_set_wait_limit(int64_t polls);

/* Tile shapes and routing of the block contractions of contractions planned
 * after this call (no counterpart in the reference, whose route-3 batching is
 * fixed by str_block): mode 0 = the fixed rule (default); 1 = autotune: at a
 * contraction's first call each candidate policy of the current precision
 * mode (FP64: the fixed rule, the 128 x 32 tile up to 64 columns, no
 * contraction splitting; split TF32: the fixed rule, tensor cores from 128 or
 * from 512 contraction indices, 9..32-column blocks on the tensor cores from
 * 256 or from 128 contraction indices) is
 * built and timed on the actual lists (result restored between the trials)
 * and the fastest is kept; the choice is cached by the plan's block-shape
 * histogram (per block contraction the binary orders of M, N, K and which
 * operands need map lookups) and reused for every plan with the same
 * histogram; 2 = always the candidate `candidate` (tests). */
int gccu_set_tuning(int64_t mode, int64_t candidate);
/* one row of 8 per tuned histogram: (block contractions, chosen candidate,
 * ms of candidates 0..5, -1 where there is none) */
int gccu_tuning_report(double* rows, int64_t maxrows, int64_t* nrows);
/* time spent making contraction plans since the engine started (no
 * counterpart in the reference): out[0] plans made, out[1..4] seconds in the
 * host planner, the string maps, the autotuner's trials and the plan builds
 * (tables, uploads, cached operand panels), of which out[5] building the
 * offset tables on the host, out[6] their upload, out[8] the descriptors,
 * tiles, job lists and allocations after it and out[7] making the cached
 * panels of frozen operands; out[9] the time inside cudaMalloc / cudaFree
 * (part of the stages above).  Host time: the device work a stage queues
 * is not waited for.  out holds 10 values. */
int gccu_plan_stats(double* out);

/* ---- statistics -----------------------------------------------------------
 * dgemm shape statistics in the reference's accounting
 * (contract/contr_blk1blk2_blocked_mm.f:454-460): [calls, sum dim1,
 * sum dim1^2, sum dim2, sum dim2^2, sum cnt, sum cnt^2, flops] accumulated
 * over the planned block contractions since the last reset, and the number of
 * kernel launches issued. */
int gccu_stats(double* stats8, int64_t* launches);
int gccu_reset_stats(void);

/* ---- timing (replaces the atim_cs timers of crout/atim.c and the
 * contr_times counters, include/contr_times.h) --------------------------------
 * CUDA events recorded on the engine's stream in slots 0..63 */
int gccu_event_record(int64_t slot);
int gccu_event_elapsed(int64_t slot_a, int64_t slot_b, double* ms);
/* per-contraction kernel timing: while enabled every [CONTR] launch is
 * bracketed by events on the engine's stream.  The report synchronises and
 * returns one row per planned contraction that ran: (flops per call,
 * calls, total kernel ms, block contractions, tiles, of which ms in the
 * operand gathers), then resets the accumulated times. */
int gccu_profile(int64_t enable);
int gccu_profile_report(double* rows, int64_t maxrows, int64_t* nrows);

#ifdef __cplusplus
}
#endif
#endif
