/*
 * orc_tree.c -- oracle restatement of the reference's tree and list construction
 * (test infrastructure only).
 *
 *   get_bounds            build_tree.h:20-35 (build_non_adaptive_tree.h:17-32)
 *   sort_bodies           build_tree.h:49-77 (non-adaptive: build_non_adaptive_tree.h:46-87)
 *   build_tree (adaptive) build_tree.h:80-199, balance_tree build_tree.h:209-359
 *   build_tree (uniform)  build_non_adaptive_tree.h:90-194
 *   keys                  hilbert.h:15-107, 115-195, 404-412 (EXAFMM_HILBERT == 0: Morton)
 *   relative-position LUT geometry.h:143-215
 *   set_colleagues        build_list.h:146-197
 *   build_list            build_list.h:16-138 (NON_ADAPTIVE variant when depth >= 0)
 *
 * The recursion keeps the reference's ping-pong of the body buffers so that the
 * rebuild after balancing starts from the same partially sorted body order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "orc.h"

typedef struct {
  double X[3];
  int ibody;
} body;

typedef struct {
  int idx, level, is_leaf, nsrcs, ntrgs, parent, octant, child0;
  double x[3], r;
  uint64_t key;
} node;

typedef struct {
  uint64_t* a;
  size_t n, cap;
} kset;

struct orc_tree {
  int nsrc, ntrg, ncrit, depth, nsurf, nonadaptive;
  double x0[3], r0;
  node* nodes;
  int nnodes, cap;
  int *leafs, nleafs, *nonleafs, nnonleafs;
  int *src_perm, nsp, *trg_perm, ntp;
  int* colleagues;
  int* m2l;
  int64_t *p2p_off, *m2p_off, *p2l_off;
  int *p2p, *m2p, *p2l;
  int64_t np2p, nm2p, np2l;
};

/* ---------------- key sets (std::set<uint64_t> semantics) ---------------- */
static void ks_push(kset* s, uint64_t v) {
  if (s->n == s->cap) {
    s->cap = s->cap ? 2 * s->cap : 64;
    s->a = (uint64_t*)realloc(s->a, s->cap * sizeof(uint64_t));
  }
  s->a[s->n++] = v;
}
static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}
static void ks_finalize(kset* s) {
  if (!s->n) return;
  qsort(s->a, s->n, sizeof(uint64_t), cmp_u64);
  size_t w = 1;
  for (size_t i = 1; i < s->n; i++)
    if (s->a[i] != s->a[w - 1]) s->a[w++] = s->a[i];
  s->n = w;
}
static int ks_has(const kset* s, uint64_t v) {
  size_t lo = 0, hi = s->n;
  while (lo < hi) {
    size_t m = (lo + hi) / 2;
    if (s->a[m] < v) lo = m + 1;
    else hi = m;
  }
  return lo < s->n && s->a[lo] == v;
}
static void ks_free(kset* s) { free(s->a); s->a = NULL; s->n = s->cap = 0; }

/* ---------------- Morton keys with level offset (hilbert.h) ---------------- */
static uint64_t level_offset(int level) { return (((uint64_t)1 << 3 * level) - 1) / 7; }
static int get_level(uint64_t i) {
  int level = -1;
  uint64_t offset = 0;
  while (i >= offset) {
    level++;
    offset += (uint64_t)1 << 3 * level;
  }
  return level;
}
static uint64_t get_parent(uint64_t i) {
  int level = get_level(i);
  return (i - level_offset(level)) / 8 + level_offset(level - 1);
}
static uint64_t get_child(uint64_t i) {
  int level = get_level(i);
  return (i - level_offset(level)) * 8 + level_offset(level + 1);
}
static uint64_t get_key(const int iX[3], int level) {
  uint64_t i = 0;
  for (int l = 0; l < level; l++) {
    i |= ((uint64_t)iX[2] & (uint64_t)1 << l) << 2 * l;
    i |= ((uint64_t)iX[1] & (uint64_t)1 << l) << (2 * l + 1);
    i |= ((uint64_t)iX[0] & (uint64_t)1 << l) << (2 * l + 2);
  }
  return i + level_offset(level);
}
static void get_3d_index_key(uint64_t i, int iX[3]) {
  int level = get_level(i);
  i -= level_offset(level);
  iX[0] = iX[1] = iX[2] = 0;
  for (int l = 0; l < level; l++) {
    iX[2] |= (int)((i & (uint64_t)1 << 3 * l) >> 2 * l);
    iX[1] |= (int)((i & (uint64_t)1 << (3 * l + 1)) >> (2 * l + 1));
    iX[0] |= (int)((i & (uint64_t)1 << (3 * l + 2)) >> (2 * l + 2));
  }
}
static void get_3d_index_x(const double X[3], int level, const double x0[3], double r0, int iX[3]) {
  double dx = 2 * r0 / (1 << level);
  for (int d = 0; d < 3; d++) iX[d] = (int)floor((X[d] - (x0[d] - r0)) / dx);
}

/* ---------------- relative-position tables (geometry.h:143-215) ---------------- */
enum { M2M_T = 0, L2L_T, M2LH_T, M2L_T, P2P0_T, P2P1_T, P2P2_T, M2P_T, P2L_T, NTYPES };
static int HASH_LUT[NTYPES][2000];
static int REL_COUNT[NTYPES];
static int rel_ready = 0;
static int hash3(const int c[3]) {
  const int n = 5;
  return ((c[2] + n) * (2 * n) + (c[1] + n)) * (2 * n) + (c[0] + n);
}
static void init_rel(int max_r, int min_r, int step, int t) {
  for (int i = 0; i < 2000; i++) HASH_LUT[t][i] = -1;
  int cnt = 0;
  for (int k = -max_r; k <= max_r; k += step)
    for (int j = -max_r; j <= max_r; j += step)
      for (int i = -max_r; i <= max_r; i += step)
        if (abs(i) >= min_r || abs(j) >= min_r || abs(k) >= min_r) {
          int c[3] = {i, j, k};
          HASH_LUT[t][hash3(c)] = cnt++;
        }
  REL_COUNT[t] = cnt;
}
static void init_rel_all(void) {
  if (rel_ready) return;
  init_rel(1, 1, 2, M2M_T);
  init_rel(1, 1, 2, L2L_T);
  init_rel(3, 3, 2, P2P0_T);
  init_rel(1, 0, 1, P2P1_T);
  init_rel(3, 3, 2, P2P2_T);
  init_rel(3, 2, 1, M2LH_T);
  init_rel(1, 1, 1, M2L_T);
  init_rel(5, 5, 2, M2P_T);
  init_rel(5, 5, 2, P2L_T);
  rel_ready = 1;
}

/* ---------------- tree construction ---------------- */
static int new_nodes(orc_tree* t, int k) {
  if (t->nnodes + k > t->cap) {
    t->cap = (t->nnodes + k) * 2;
    t->nodes = (node*)realloc(t->nodes, (size_t)t->cap * sizeof(node));
  }
  int first = t->nnodes;
  memset(t->nodes + first, 0, (size_t)k * sizeof(node));
  t->nnodes += k;
  return first;
}
static void push_int(int** a, int* n, int v) {
  if ((*n & (*n - 1)) == 0) *a = (int*)realloc(*a, (size_t)(*n ? 2 * *n : 1) * sizeof(int));
  (*a)[(*n)++] = v;
}

static int octant_of(const double x[3], const double X[3]) {
  return (x[0] > X[0]) + ((x[1] > X[1]) << 1) + ((x[2] > X[2]) << 2);
}

/* build_tree.h:49-77: stable 8-way counting sort of bodies[begin,end) into buffer */
static void sort_bodies(const double X[3], const body* bodies, body* buffer, int begin, int end, int size[8],
                        int offsets[8]) {
  for (int i = 0; i < 8; i++) size[i] = 0;
  for (int i = begin; i < end; i++) size[octant_of(bodies[i].X, X)]++;
  int offset = begin;
  for (int i = 0; i < 8; i++) {
    offsets[i] = offset;
    offset += size[i];
  }
  int counter[8];
  memcpy(counter, offsets, sizeof(counter));
  for (int i = begin; i < end; i++) buffer[counter[octant_of(bodies[i].X, X)]++] = bodies[i];
}

static void make_children(orc_tree* t, int ni, int first) {
  t->nodes[ni].child0 = first;
  for (int c = 0; c < 8; c++) {
    node* ch = &t->nodes[first + c];
    const node* pa = &t->nodes[ni];
    for (int d = 0; d < 3; d++) ch->x[d] = pa->x[d];
    ch->r = pa->r / 2;
    for (int d = 0; d < 3; d++) ch->x[d] += ch->r * (double)((((c & 1 << d) >> d) * 2) - 1);
    ch->parent = ni;
    ch->octant = c;
    ch->level = pa->level + 1;
  }
}

static void init_node(orc_tree* t, int ni, int ns, int nt) {
  node* n = &t->nodes[ni];
  n->idx = ni;
  n->nsrcs = ns;
  n->ntrgs = nt;
  n->child0 = -1;
  int iX[3];
  get_3d_index_x(n->x, n->level, t->x0, t->r0, iX);
  n->key = get_key(iX, n->level);
}

/* build_tree.h:80-166 */
static void build_adaptive(orc_tree* t, body* src, body* src_buf, int sb, int se, body* trg, body* trg_buf, int tb,
                           int te, int ni, const kset* leafkeys, int nlk, int direction) {
  init_node(t, ni, se - sb, te - tb);
  node* n = &t->nodes[ni];
  int is_leaf_key = 1;
  if (nlk) is_leaf_key = ks_has(&leafkeys[n->level], n->key);
  if (n->nsrcs <= t->ncrit && n->ntrgs <= t->ncrit && is_leaf_key) {
    n->is_leaf = 1;
    if (n->nsrcs || n->ntrgs) push_int(&t->leafs, &t->nleafs, ni);
    if (direction) {
      for (int i = sb; i < se; i++) src_buf[i] = src[i];
      for (int i = tb; i < te; i++) trg_buf[i] = trg[i];
    }
    if (nlk) {
      const body* fs = (direction ? src_buf : src) + sb;
      const body* ft = (direction ? trg_buf : trg) + tb;
      for (int i = 0; i < n->nsrcs; i++) t->src_perm[t->nsp++] = fs[i].ibody;
      for (int i = 0; i < n->ntrgs; i++) t->trg_perm[t->ntp++] = ft[i].ibody;
    }
    return;
  }
  int ssize[8], soff[8], tsize[8], toff[8];
  double X[3] = {n->x[0], n->x[1], n->x[2]};
  sort_bodies(X, src, src_buf, sb, se, ssize, soff);
  sort_bodies(X, trg, trg_buf, tb, te, tsize, toff);
  n->is_leaf = 0;
  push_int(&t->nonleafs, &t->nnonleafs, ni);
  int first = new_nodes(t, 8);
  make_children(t, ni, first);
  for (int c = 0; c < 8; c++)
    build_adaptive(t, src_buf, src, soff[c], soff[c] + ssize[c], trg_buf, trg, toff[c], toff[c] + tsize[c],
                   first + c, leafkeys, nlk, !direction);
}

static void reset_nodes(orc_tree* t) {
  t->nnodes = 0;
  t->nleafs = t->nnonleafs = 0;
  t->nsp = t->ntp = 0;
  int r = new_nodes(t, 1);
  node* root = &t->nodes[r];
  for (int d = 0; d < 3; d++) root->x[d] = t->x0[d];
  root->r = t->r0;
  root->level = 0;
  root->parent = -1;
  root->octant = 0;
}

/* build_tree.h:336-359 (with breadth_first_traversal 209-236, balance_tree 247-300, find_leaf_keys 308-323) */
static void balance(orc_tree* t, body* src, body* src_buf, body* trg, body* trg_buf) {
  int nlev = 0;
  for (int i = 0; i < t->nnodes; i++)
    if (t->nodes[i].level + 1 > nlev) nlev = t->nodes[i].level + 1;
  kset* keys = (kset*)calloc((size_t)nlev, sizeof(kset));
  kset* nonleaf = (kset*)calloc((size_t)nlev, sizeof(kset));
  for (int i = 0; i < t->nnodes; i++) {
    ks_push(&keys[t->nodes[i].level], t->nodes[i].key);
    if (!t->nodes[i].is_leaf) ks_push(&nonleaf[t->nodes[i].level], t->nodes[i].key);
  }
  for (int l = 0; l < nlev; l++) {
    ks_finalize(&keys[l]);
    ks_finalize(&nonleaf[l]);
  }
  kset* use;
  kset* bkeys = NULL;
  kset* leafkeys = NULL;
  if (t->nnodes == 1) {
    use = keys;
  } else {
    const int maxlevel = nlev - 1;
    bkeys = (kset*)calloc((size_t)nlev, sizeof(kset));
    kset S = {0}, N = {0};
    for (int l = maxlevel; l > 0; --l) {
      N.n = 0;
      for (size_t i = 0; i < nonleaf[l].n; i++) ks_push(&N, nonleaf[l].a[i]);
      for (size_t i = 0; i < S.n; i++) ks_push(&N, S.a[i]);
      ks_finalize(&N);
      S.n = 0;
      for (size_t i = 0; i < N.n; i++) {
        int iX[3];
        get_3d_index_key(N.a[i], iX);
        for (int m = -1; m <= 1; ++m)
          for (int nn = -1; nn <= 1; ++nn)
            for (int p = -1; p <= 1; ++p) {
              if (!(m || nn || p)) continue;
              int c[3] = {iX[0] + m, iX[1] + nn, iX[2] + p};
              double lim = pow(2, l);
              if (c[0] >= 0 && c[0] < lim && c[1] >= 0 && c[1] < lim && c[2] >= 0 && c[2] < lim)
                ks_push(&S, get_parent(get_key(c, l)));
            }
      }
      ks_finalize(&S);
      if (l != maxlevel) {
        for (size_t i = 0; i < N.n; i++) {
          uint64_t ch = get_child(N.a[i]);
          for (int k = 0; k < 8; ++k) ks_push(&bkeys[l + 1], ch + k);
        }
      }
    }
    ks_push(&bkeys[0], 0);
    for (int i = 1; i < 9; ++i) ks_push(&bkeys[1], (uint64_t)i);
    for (int l = 0; l < nlev; l++) ks_finalize(&bkeys[l]);
    ks_free(&S);
    ks_free(&N);
    /* find_leaf_keys */
    leafkeys = (kset*)calloc((size_t)nlev, sizeof(kset));
    for (int l = nlev - 1; l >= 1; --l) {
      kset pk = {0};
      for (size_t i = 0; i < bkeys[l - 1].n; i++) ks_push(&pk, bkeys[l - 1].a[i]);
      kset par = {0};
      for (size_t i = 0; i < bkeys[l].n; i++) ks_push(&par, get_parent(bkeys[l].a[i]));
      ks_finalize(&par);
      for (size_t i = 0; i < pk.n; i++)
        if (!ks_has(&par, pk.a[i])) ks_push(&leafkeys[l - 1], pk.a[i]);
      ks_finalize(&leafkeys[l - 1]);
      ks_free(&pk);
      ks_free(&par);
    }
    for (size_t i = 0; i < bkeys[nlev - 1].n; i++) ks_push(&leafkeys[nlev - 1], bkeys[nlev - 1].a[i]);
    ks_finalize(&leafkeys[nlev - 1]);
    use = leafkeys;
  }
  /* rebuild from the (partially sorted) body arrays, as build_tree.h:345-356 */
  memcpy(src_buf, src, sizeof(body) * (size_t)t->nsrc);
  memcpy(trg_buf, trg, sizeof(body) * (size_t)t->ntrg);
  reset_nodes(t);
  build_adaptive(t, src, src_buf, 0, t->nsrc, trg, trg_buf, 0, t->ntrg, 0, use, nlev, 0);
  t->depth = nlev - 1;
  for (int l = 0; l < nlev; l++) {
    ks_free(&keys[l]);
    ks_free(&nonleaf[l]);
    if (bkeys) ks_free(&bkeys[l]);
    if (leafkeys) ks_free(&leafkeys[l]);
  }
  free(keys);
  free(nonleaf);
  free(bkeys);
  free(leafkeys);
}

/* build_non_adaptive_tree.h:46-87: in-place stable octant sort */
static void sort_inplace(const double X[3], body* b, int begin, int end, int size[8], int offsets[8]) {
  for (int i = 0; i < 8; i++) {
    size[i] = 0;
    offsets[i] = begin;
  }
  if (end == begin) return;
  for (int i = begin; i < end; i++) size[octant_of(b[i].X, X)]++;
  int counter[8], offset = begin;
  for (int i = 0; i < 8; i++) {
    offsets[i] = offset;
    offset += size[i];
    counter[i] = offsets[i] - begin;
  }
  body* buf = (body*)malloc(sizeof(body) * (size_t)(end - begin));
  for (int i = begin; i < end; i++) buf[counter[octant_of(b[i].X, X)]++] = b[i];
  memcpy(b + begin, buf, sizeof(body) * (size_t)(end - begin));
  free(buf);
}

/* build_non_adaptive_tree.h:90-166 */
static void build_uniform(orc_tree* t, body* src, int sb, int se, body* trg, int tb, int te, int ni) {
  init_node(t, ni, se - sb, te - tb);
  node* n = &t->nodes[ni];
  if (n->nsrcs == 0 && n->ntrgs == 0) {
    n->is_leaf = 1;
    return;
  }
  if (n->level == t->depth) {
    n->is_leaf = 1;
    push_int(&t->leafs, &t->nleafs, ni);
    for (int i = sb; i < se; i++) t->src_perm[t->nsp++] = src[i].ibody;
    for (int i = tb; i < te; i++) t->trg_perm[t->ntp++] = trg[i].ibody;
    return;
  }
  int ssize[8], soff[8], tsize[8], toff[8];
  double X[3] = {n->x[0], n->x[1], n->x[2]};
  sort_inplace(X, src, sb, se, ssize, soff);
  sort_inplace(X, trg, tb, te, tsize, toff);
  n->is_leaf = 0;
  push_int(&t->nonleafs, &t->nnonleafs, ni);
  int first = new_nodes(t, 8);
  make_children(t, ni, first);
  for (int c = 0; c < 8; c++)
    build_uniform(t, src, soff[c], soff[c] + ssize[c], trg, toff[c], toff[c] + tsize[c], first + c);
}

/* ---------------- colleagues and lists (build_list.h) ---------------- */
static void set_colleagues(orc_tree* t, int ni) {
  node* n = &t->nodes[ni];
  int* col = &t->colleagues[27 * (size_t)ni];
  for (int i = 0; i < 27; i++) col[i] = -1;
  if (n->level == 0) {
    col[13] = ni;
  } else {
    const int* pcol = &t->colleagues[27 * (size_t)n->parent];
    const int l = n->octant;
    for (int i = 0; i < 27; ++i) {
      int cg = pcol[i];
      if (cg >= 0 && !t->nodes[cg].is_leaf) {
        for (int j = 0; j < 8; ++j) {
          int child = t->nodes[cg].child0 + j;
          int flag = 1, a = 1, b = 1, new_idx = 0;
          for (int k = 0; k < 3; ++k) {
            int idx_diff = (((i / b) % 3) - 1) * 2 + ((j / a) % 2) - ((l / a) % 2);
            if (-1 > idx_diff || idx_diff > 1) flag = 0;
            new_idx += (idx_diff + 1) * b;
            a *= 2;
            b *= 3;
          }
          if (flag) col[new_idx] = child;
        }
      }
    }
  }
  if (!n->is_leaf)
    for (int c = 0; c < 8; ++c) set_colleagues(t, t->nodes[ni].child0 + c);
}

typedef struct {
  int* a;
  int64_t n, cap;
} ivec;
static void iv_push(ivec* v, int x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 256;
    v->a = (int*)realloc(v->a, (size_t)v->cap * sizeof(int));
  }
  v->a[v->n++] = x;
}

static void build_lists(orc_tree* t) {
  const int nn = t->nnodes;
  ivec P2P = {0}, M2P = {0}, P2L = {0};
  t->p2p_off = (int64_t*)calloc((size_t)nn + 1, sizeof(int64_t));
  t->m2p_off = (int64_t*)calloc((size_t)nn + 1, sizeof(int64_t));
  t->p2l_off = (int64_t*)calloc((size_t)nn + 1, sizeof(int64_t));
  t->m2l = (int*)malloc(sizeof(int) * 26 * (size_t)nn);
  for (int ni = 0; ni < nn; ni++) {
    node* n = &t->nodes[ni];
    t->p2p_off[ni] = P2P.n;
    t->m2p_off[ni] = M2P.n;
    t->p2l_off[ni] = P2L.n;
    int* m2l = &t->m2l[26 * (size_t)ni];
    for (int k = 0; k < 26; k++) m2l[k] = -1;
    const int* col = &t->colleagues[27 * (size_t)ni];
    int rc[3];
    /* build_list_parent_level (16-43) */
    if (n->parent >= 0) {
      const int* pcol = &t->colleagues[27 * (size_t)n->parent];
      for (int i = 0; i < 27; i++) {
        int pc = pcol[i];
        if (pc >= 0 && t->nodes[pc].is_leaf) {
          rc[0] = (i % 3) * 4 - 4 - (n->octant & 1 ? 2 : 0) + 1;
          rc[1] = ((i / 3) % 3) * 4 - 4 - (n->octant & 2 ? 2 : 0) + 1;
          rc[2] = ((i / 9) % 3) * 4 - 4 - (n->octant & 4 ? 2 : 0) + 1;
          int h = hash3(rc);
          if (n->is_leaf && HASH_LUT[P2P0_T][h] >= 0) iv_push(&P2P, pc);
          if (HASH_LUT[P2L_T][h] >= 0) {
            if (n->is_leaf && n->ntrgs <= t->nsurf) iv_push(&P2P, pc);
            else iv_push(&P2L, pc);
          }
        }
      }
    }
    /* build_list_current_level (52-74) */
    for (int i = 0; i < 27; i++) {
      int c = col[i];
      if (c >= 0) {
        rc[0] = (i % 3) - 1;
        rc[1] = ((i / 3) % 3) - 1;
        rc[2] = ((i / 9) % 3) - 1;
        int h = hash3(rc);
        if (t->nodes[c].is_leaf && n->is_leaf) {
          if (HASH_LUT[P2P1_T][h] >= 0) iv_push(&P2P, c);
        } else if (!t->nodes[c].is_leaf && !n->is_leaf) {
          int idx2 = HASH_LUT[M2L_T][h];
          if (idx2 >= 0) m2l[idx2] = c;
        }
      }
    }
    /* build_list_child_level (84-114), gated by ntrgs in the NON_ADAPTIVE build (131-136) */
    if (n->is_leaf && (!t->nonadaptive || n->ntrgs)) {
      for (int i = 0; i < 27; i++) {
        int c = col[i];
        if (c >= 0 && !t->nodes[c].is_leaf) {
          for (int j = 0; j < 8; j++) {
            int cc = t->nodes[c].child0 + j;
            rc[0] = (i % 3) * 4 - 4 + (j & 1 ? 2 : 0) - 1;
            rc[1] = ((i / 3) % 3) * 4 - 4 + (j & 2 ? 2 : 0) - 1;
            rc[2] = ((i / 9) % 3) * 4 - 4 + (j & 4 ? 2 : 0) - 1;
            int h = hash3(rc);
            if (HASH_LUT[P2P2_T][h] >= 0) iv_push(&P2P, cc);
            if (HASH_LUT[M2P_T][h] >= 0) {
              if (t->nodes[cc].is_leaf && t->nodes[cc].nsrcs <= t->nsurf) iv_push(&P2P, cc);
              else iv_push(&M2P, cc);
            }
          }
        }
      }
    }
  }
  t->p2p_off[nn] = P2P.n;
  t->m2p_off[nn] = M2P.n;
  t->p2l_off[nn] = P2L.n;
  t->p2p = P2P.a;
  t->np2p = P2P.n;
  t->m2p = M2P.a;
  t->nm2p = M2P.n;
  t->p2l = P2L.a;
  t->np2l = P2L.n;
}

/* ---------------- public entry points ---------------- */
orc_tree* orc_build(int nsrc, const double* sxyz, int ntrg, const double* txyz, int ncrit, int depth, int nsurf) {
  init_rel_all();
  orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
  if (!t) return NULL;
  t->nsrc = nsrc;
  t->ntrg = ntrg;
  t->ncrit = ncrit;
  t->nsurf = nsurf;
  t->nonadaptive = depth >= 0;
  body* src = (body*)malloc(sizeof(body) * (size_t)(nsrc > 0 ? nsrc : 1));
  body* trg = (body*)malloc(sizeof(body) * (size_t)(ntrg > 0 ? ntrg : 1));
  body* src_buf = (body*)malloc(sizeof(body) * (size_t)(nsrc > 0 ? nsrc : 1));
  body* trg_buf = (body*)malloc(sizeof(body) * (size_t)(ntrg > 0 ? ntrg : 1));
  for (int i = 0; i < nsrc; i++) {
    for (int d = 0; d < 3; d++) src[i].X[d] = sxyz[3 * i + d];
    src[i].ibody = i;
  }
  for (int i = 0; i < ntrg; i++) {
    for (int d = 0; d < 3; d++) trg[i].X[d] = txyz[3 * i + d];
    trg[i].ibody = i;
  }
  /* get_bounds (build_tree.h:20-35) */
  double Xmin[3], Xmax[3];
  for (int d = 0; d < 3; d++) Xmin[d] = Xmax[d] = src[0].X[d];
  for (int b = 0; b < nsrc; b++)
    for (int d = 0; d < 3; d++) {
      Xmin[d] = src[b].X[d] < Xmin[d] ? src[b].X[d] : Xmin[d];
      Xmax[d] = src[b].X[d] > Xmax[d] ? src[b].X[d] : Xmax[d];
    }
  for (int b = 0; b < ntrg; b++)
    for (int d = 0; d < 3; d++) {
      Xmin[d] = trg[b].X[d] < Xmin[d] ? trg[b].X[d] : Xmin[d];
      Xmax[d] = trg[b].X[d] > Xmax[d] ? trg[b].X[d] : Xmax[d];
    }
  double a = 0, b2 = 0;
  for (int d = 0; d < 3; d++) t->x0[d] = (Xmax[d] + Xmin[d]) / 2;
  a = t->x0[0] - Xmin[0];
  for (int d = 1; d < 3; d++) a = a > t->x0[d] - Xmin[d] ? a : t->x0[d] - Xmin[d];
  b2 = Xmax[0] - t->x0[0];
  for (int d = 1; d < 3; d++) b2 = b2 > Xmax[d] - t->x0[d] ? b2 : Xmax[d] - t->x0[d];
  t->r0 = fmax(a, b2);
  t->r0 *= 1.00001;

  t->src_perm = (int*)malloc(sizeof(int) * (size_t)(nsrc > 0 ? nsrc : 1));
  t->trg_perm = (int*)malloc(sizeof(int) * (size_t)(ntrg > 0 ? ntrg : 1));
  reset_nodes(t);
  if (depth >= 0) {
    t->depth = depth;
    build_uniform(t, src, 0, nsrc, trg, 0, ntrg, 0);
  } else {
    memcpy(src_buf, src, sizeof(body) * (size_t)nsrc);
    memcpy(trg_buf, trg, sizeof(body) * (size_t)ntrg);
    build_adaptive(t, src, src_buf, 0, nsrc, trg, trg_buf, 0, ntrg, 0, NULL, 0, 0);
    balance(t, src, src_buf, trg, trg_buf);
  }
  free(src);
  free(trg);
  free(src_buf);
  free(trg_buf);
  t->colleagues = (int*)malloc(sizeof(int) * 27 * (size_t)t->nnodes);
  set_colleagues(t, 0);
  build_lists(t);
  return t;
}

void orc_free(orc_tree* t) {
  if (!t) return;
  free(t->nodes);
  free(t->leafs);
  free(t->nonleafs);
  free(t->src_perm);
  free(t->trg_perm);
  free(t->colleagues);
  free(t->m2l);
  free(t->p2p_off);
  free(t->m2p_off);
  free(t->p2l_off);
  free(t->p2p);
  free(t->m2p);
  free(t->p2l);
  free(t);
}

void orc_sizes(const orc_tree* t, int64_t* s) {
  s[0] = t->nnodes;
  s[1] = t->nleafs;
  s[2] = t->nnonleafs;
  s[3] = t->depth;
  s[4] = t->np2p;
  s[5] = t->nm2p;
  s[6] = t->np2l;
  s[7] = t->nsurf;
}

void orc_dump(const orc_tree* t, double* geo, uint64_t* key, int32_t* ni, double* nx, int32_t* leafs,
              int32_t* nonleafs, int32_t* src_perm, int32_t* trg_perm, int32_t* colleagues, int32_t* m2l,
              int64_t* p2p_off, int32_t* p2p, int64_t* m2p_off, int32_t* m2p, int64_t* p2l_off, int32_t* p2l) {
  for (int d = 0; d < 3; d++) geo[d] = t->x0[d];
  geo[3] = t->r0;
  for (int i = 0; i < t->nnodes; i++) {
    const node* n = &t->nodes[i];
    key[i] = n->key;
    int32_t v[8] = {n->idx, n->level, n->is_leaf, n->nsrcs, n->ntrgs, n->parent, n->octant,
                    n->is_leaf ? -1 : n->child0};
    memcpy(&ni[8 * (size_t)i], v, sizeof(v));
    for (int d = 0; d < 3; d++) nx[4 * (size_t)i + d] = n->x[d];
    nx[4 * (size_t)i + 3] = n->r;
  }
  memcpy(leafs, t->leafs, sizeof(int) * (size_t)t->nleafs);
  memcpy(nonleafs, t->nonleafs, sizeof(int) * (size_t)t->nnonleafs);
  memcpy(src_perm, t->src_perm, sizeof(int) * (size_t)t->nsp);
  memcpy(trg_perm, t->trg_perm, sizeof(int) * (size_t)t->ntp);
  memcpy(colleagues, t->colleagues, sizeof(int) * 27 * (size_t)t->nnodes);
  memcpy(m2l, t->m2l, sizeof(int) * 26 * (size_t)t->nnodes);
  memcpy(p2p_off, t->p2p_off, sizeof(int64_t) * ((size_t)t->nnodes + 1));
  memcpy(m2p_off, t->m2p_off, sizeof(int64_t) * ((size_t)t->nnodes + 1));
  memcpy(p2l_off, t->p2l_off, sizeof(int64_t) * ((size_t)t->nnodes + 1));
  if (t->np2p) memcpy(p2p, t->p2p, sizeof(int) * (size_t)t->np2p);
  if (t->nm2p) memcpy(m2p, t->m2p, sizeof(int) * (size_t)t->nm2p);
  if (t->np2l) memcpy(p2l, t->p2l, sizeof(int) * (size_t)t->np2l);
}
