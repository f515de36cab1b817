/*
 * orc.h -- the oracle: a CPU restatement of exafmm-t's setup and near-field
 * algorithms, written in plain C for the tests (test infrastructure only; the
 * product never links it).  Each function cites the reference lines it restates.
 *
 * Tree output format (shared with oracle/ref_capi.cpp so the two can be diffed):
 *   nodes are numbered in the reference's allocation order (build_tree.h:86,148)
 *   ni[8*i + {0..7}] = idx, level, is_leaf, nsrcs, ntrgs, parent, octant, first child
 *   nx[4*i + {0..3}] = centre x, y, z, radius r
 */
#ifndef XFMM_ORC_H
#define XFMM_ORC_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_tree orc_tree;

/* Build the tree (adaptive + 2:1 balance when depth < 0, else non-adaptive to `depth`),
 * colleagues and interaction lists.  nsurf feeds the P2P/P2L and M2P/P2P switches
 * (build_list.h:36-39, 105-110).  Returns NULL on allocation failure. */
orc_tree* orc_build(int nsrc, const double* sxyz, int ntrg, const double* txyz, int ncrit, int depth, int nsurf);
void orc_free(orc_tree* t);
/* sizes: nnodes, nleafs, nnonleafs, depth, np2p, nm2p, np2l, 0 */
void orc_sizes(const orc_tree* t, int64_t* s);
void orc_dump(const orc_tree* t, double* geo, uint64_t* key, int32_t* ni, double* nx, int32_t* leafs,
              int32_t* nonleafs, int32_t* src_perm, int32_t* trg_perm, int32_t* colleagues, int32_t* m2l,
              int64_t* p2p_off, int32_t* p2p, int64_t* m2p_off, int32_t* m2p, int64_t* p2l_off, int32_t* p2l);

/* Scalar FP64 kernels: kernel 0 Laplace, 1 modified Helmholtz (k real), 2 Helmholtz (complex k).
 * Values/outputs are interleaved complex for kernel 2.  Output is accumulated. */
void orc_gradient_p2p(int kernel, double k_re, double k_im, int ns, const double* sxyz, const double* sq, int nt,
                      const double* txyz, double* out);
void orc_potential_p2p(int kernel, double k_re, double k_im, int ns, const double* sxyz, const double* sq, int nt,
                       const double* txyz, double* out);

#ifdef __cplusplus
}
#endif
#endif
