/*
 * ORACLE -- CPU restatement of GeCCo's blocked tensor-contraction path.
 *
 * This is TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it, and only as the
 * checker or the timed CPU baseline.  The product (libgccu) never links it.
 *
 * Each routine restates one reference routine (file:line given at the
 * definition in oracle.cpp).  Parity is pinned by golden values taken from the
 * reference's own regression output (tests/golden/), see oracle.cpp header.
 *
 * Conventions at this interface: integers are int64_t, reals double, indices
 * and irreps are 1-based like the reference, occupations are [2][4] arrays
 * (C row then A row; columns H,P,V,X).
 */
#ifndef GECCO_ORACLE_H
#define GECCO_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_ctx ora_ctx;

/* orbital space: nsym irreps (1,2,4,8); norb[t*8+g] = active orbitals of
 * hpvx type t (0=H,1=P,2=V,3=X) in irrep g (0-based) */
ora_ctx* ora_create(int64_t nsym, const int64_t* norb);
void     ora_destroy(ora_ctx*);
const char* ora_last_error(void);

/* string enumeration of graph (type,nel) in reference order for block
 * (idxms, gam) -- strings/next_string.f; writes orb/spn (nel per string) */
int64_t ora_graph_nstr(ora_ctx*, int64_t type, int64_t nel, int64_t idxms, int64_t gam);
int64_t ora_graph_strings(ora_ctx*, int64_t type, int64_t nel, int64_t idxms,
                          int64_t gam, int64_t* orb, int64_t* spn);

/* one block of the signed (str1,str2)->str12 map -- strings/set_strmap_kernel.f */
int64_t ora_strmap_block(ora_ctx*, int64_t type, int64_t nel1, int64_t nel2,
                         int64_t idxms1, int64_t idxms2, int64_t gam1, int64_t gam2,
                         int64_t* map /* nstr1*nstr2, str1 fastest */);

/* operator = list of occupation classes occ[nblk][2][4] */
int64_t ora_define_op(ora_ctx*, const int64_t* occ, int64_t nblk);
/* joined operator: occ holds nblk*nj occupations, vertices of a class consecutive */
int64_t ora_define_op_joined(ora_ctx*, const int64_t* occ, int64_t nj, int64_t nblk);
/* ME list layout -- operators/set_op_dim2.f; returns list id, *len = len_op */
int64_t ora_define_list(ora_ctx*, int64_t op, int64_t gamt, int64_t mst,
                        int64_t absym, int64_t* len);
/* layout tables of a list block: off/len per occupation class */
int ora_list_block(ora_ctx*, int64_t list, int64_t iblk, int64_t* off, int64_t* len);
/* flattened distribution table of a list: rows of
 * (iblk, idxmsa, gama, idxdis, offset, length, ld, did) -> returns row count */
int64_t ora_list_dists(ora_ctx*, int64_t list, int64_t* rows, int64_t maxrows);

/* binary contraction -- contract/contr_op1op2_wmaps_c.f
 * route 2: contract/contr_blk1blk2_wmaps_c.f (scalar loops)
 * route 3: contract/contr_blk1blk2_blocked_mm.f (gather / dgemm / scatter)
 * iblk12 = 0 means scalar result (written to/accumulated in *xret).
 * stats (may be NULL): [ncalls, sum dim1, sum dim1^2, sum dim2, sum dim2^2,
 *                       sum cnt, sum cnt^2, flops] of the route-3 dgemm calls */
int ora_contract(ora_ctx*, int64_t route,
                 int64_t list1, int64_t iblk1, const double* x1,
                 int64_t list2, int64_t iblk2, const double* x2,
                 int64_t list12, int64_t iblk12, double* x12,
                 const int64_t* occ_ex1, const int64_t* occ_ex2,
                 const int64_t* occ_cnt,
                 double fact, int64_t update, int64_t use_tr,
                 int64_t str_block, int64_t cnt_block,
                 double* xret, double* stats);
/* the same with operands used transposed (tra_op1, tra_op2, tra_op1op2 of
 * contract/contr_op1op2_wmaps_c.f): occ_ex1/occ_ex2/occ_cnt describe the
 * contraction of the adjoint classes */
int ora_contract_t(ora_ctx*, int64_t route,
                   int64_t list1, int64_t iblk1, const double* x1,
                   int64_t list2, int64_t iblk2, const double* x2,
                   int64_t list12, int64_t iblk12, double* x12,
                   const int64_t* occ_ex1, const int64_t* occ_ex2,
                   const int64_t* occ_cnt,
                   double fact, int64_t update, int64_t use_tr,
                   int64_t tra_op1, int64_t tra_op2, int64_t tra_res,
                   double* xret);

/* spin-flip symmetrisation of a result block -- contract/sym_ab_blk.f */
/* reorder (reo_op_wmaps_c / reo_blk_wmaps_c) of class iblk_ori of list_ori
 * into class iblk_reo of list_reo: shift s (occ_shift[8*s..]) moves from
 * vertex from_vtx[s] to to_vtx[s] (1-based); xreo (whole list) updated */
int ora_reorder(ora_ctx*, int64_t list_ori, int64_t iblk_ori, const double* xori,
                int64_t list_reo, int64_t iblk_reo, double* xreo, int64_t nshift,
                const int64_t* occ_shift, const int64_t* from_vtx, const int64_t* to_vtx,
                double fac, int64_t sign_reo, int64_t update);
/* partial trace (trace_op / trace_op_blk): xres (whole list) +=
 * fac * sum_J xop(IC*J, IA*J), J of occupation occ_cnt on both sides */
int ora_trace(ora_ctx*, int64_t list_op, int64_t iblk_op, const double* xop,
              int64_t list_res, int64_t iblk_res, double* xres, const int64_t* occ_cnt,
              double fac, int64_t update);
int ora_sym_ab_blk(ora_ctx*, int64_t list, int64_t iblk, double* x,
                   double prefac, double relfac);

/* spin projection of a whole list onto its singlet part, in place --
 * contract/spin_prj_list.f with contract/spin_prj_blk.f; s2 must be 0;
 * xnorm2 (may be NULL) receives the squared norm of every projected class */
int ora_spin_prj_list(ora_ctx*, int64_t list, int64_t s2, double* x, double* xnorm2);

/* route-3 dgemm through an ILP64 BLAS (e.g. the OpenBLAS bundled with numpy)
 * instead of the plain loop; nthreads > 0 sets the BLAS thread count */
int ora_set_blas(const char* path, int64_t nthreads);
/* CPU-baseline sampling: execute only every stride-th long-operand batch of
 * route 3 (and the short-operand gathers those batches need); the report
 * gives [seconds in short-operand gathers, seconds in executed batches,
 * batches total, batches executed, short gathers total, short gathers
 * executed] since the last ora_sampling call */
void ora_sampling(int64_t stride);
void ora_sampling_report(double* out6);

/* add_opblk (in-core branch) -- contract/add_opblk.f:299-307 */
int ora_add_opblk(double* xnorm2, int64_t type, double fac, const double* xin,
                  double* xout, int64_t len, int64_t reset);
/* diavc -- baserout/diavc.f:31-35 */
void ora_diavc(double* out, const double* in, double fac, const double* diag,
               double shift, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
