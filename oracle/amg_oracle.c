/*
 * amg_oracle.c -- TEST INFRASTRUCTURE ONLY: a CPU restatement of the
 * reference solver (liuzhengqi1996/blood_network, C_amg1), written from the
 * reference's behaviour so the CUDA library can be checked against it.
 * Nothing in the product links this file.  Each routine names the reference
 * file:line it restates; operation order (sequential sums, separate multiply
 * and add, in-place updates) follows the reference so results are
 * bit-identical to it.  Pinned against fixtures generated from the compiled
 * reference (tests/golden/).
 */
#include "amg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define C_PT 1
#define F_PT (-1)
#define UNDEC 0

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

void orc_csr_free(orc_csr* a) {
  if (!a) return;
  free(a->ia);
  free(a->ja);
  free(a->val);
  memset(a, 0, sizeof(*a));
}

static void csr_alloc(orc_csr* a, int n, int m, int nnz) {
  a->n = n;
  a->m = m;
  a->nnz = nnz;
  a->ia = (int*)xcalloc((size_t)n + 1, sizeof(int));
  a->ja = (int*)xcalloc((size_t)nnz, sizeof(int));
  a->val = (double*)xcalloc((size_t)nnz, sizeof(double));
}

/* Stable counting-sort transpose: agg_lib.h:120-183. */
void orc_transpose(const orc_csr* a, orc_csr* t) {
  csr_alloc(t, a->m, a->n, a->nnz);
  for (int k = 0; k < a->nnz; k++) t->ia[a->ja[k] + 1]++;
  for (int j = 0; j < a->m; j++) t->ia[j + 1] += t->ia[j];
  int* fill = (int*)xcalloc((size_t)a->m, sizeof(int));
  for (int i = 0; i < a->n; i++)
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      int j = a->ja[k];
      int q = t->ia[j] + fill[j]++;
      t->ja[q] = i;
      t->val[q] = a->val ? a->val[k] : 0.0;
    }
  free(fill);
}

/* Sparse add in the reference's entry order, then scaling:
 * agg_lib.h:186-243 (+ the "*= 0.5" of amg_wrapper.c:59-76). */
void orc_add_scaled(const orc_csr* a, const orc_csr* b, double scale, orc_csr* c) {
  const int n = a->n, m = a->m;
  int* mark = (int*)xcalloc((size_t)m, sizeof(int));
  for (int j = 0; j < m; j++) mark[j] = -1;
  int total = 0;
  for (int i = 0; i < n; i++) {
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      mark[a->ja[k]] = i;
      total++;
    }
    for (int k = b->ia[i]; k < b->ia[i + 1]; k++)
      if (mark[b->ja[k]] != i) {
        mark[b->ja[k]] = i;
        total++;
      }
  }
  csr_alloc(c, n, m, total);
  for (int j = 0; j < m; j++) mark[j] = -1;
  double* w = (double*)xcalloc((size_t)m, sizeof(double));
  int pos = 0;
  for (int i = 0; i < n; i++) {
    const int start = pos;
    c->ia[i] = start;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      int col = a->ja[k];
      mark[col] = pos;
      c->ja[pos++] = col;
      w[col] = a->val[k];
    }
    for (int k = b->ia[i]; k < b->ia[i + 1]; k++) {
      int col = b->ja[k];
      if (mark[col] >= start) {
        w[col] += b->val[k];
      } else {
        mark[col] = pos;
        c->ja[pos++] = col;
        w[col] = b->val[k];
      }
    }
    for (int q = start; q < pos; q++) {
      c->val[q] = w[c->ja[q]];
      w[c->ja[q]] = 0.0;
    }
  }
  c->ia[n] = pos;
  c->nnz = pos;
  for (int q = 0; q < pos; q++) c->val[q] *= scale;
  free(mark);
  free(w);
}

void orc_symmetrize(const orc_csr* a, orc_csr* out) {
  orc_csr t;
  orc_transpose(a, &t);
  orc_add_scaled(a, &t, 0.5, out);
  orc_csr_free(&t);
}

/* Strength of connection: rs_classical.c:30-88. */
void orc_strength(const orc_csr* a, double theta, orc_csr* s, int* max_lam) {
  const int n = a->n;
  double* thr = (double*)xcalloc((size_t)n, sizeof(double));
  int ml = 0;
  for (int i = 0; i < n; i++) {
    double mx = 0.0;
    int len = a->ia[i + 1] - a->ia[i];
    if (len > ml) ml = len;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      if (a->ja[k] == i) continue;
      double v = -(a->val[k]);
      if (v > mx) mx = v;
    }
    thr[i] = theta * mx;
  }
  *max_lam = ml < 1 ? 1 : ml;
  int cnt = 0;
  for (int i = 0; i < n; i++)
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++)
      if (a->ja[k] != i && -(a->val[k]) >= thr[i]) cnt++;
  csr_alloc(s, n, a->m, cnt);
  int p = 0;
  for (int i = 0; i < n; i++) {
    s->ia[i] = p;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++)
      if (a->ja[k] != i && -(a->val[k]) >= thr[i]) {
        s->ja[p] = a->ja[k];
        s->val[p] = a->val[k];
        p++;
      }
  }
  s->ia[n] = p;
  free(thr);
}

/* ---- doubly linked bucket lists for the RS greedy (rs_classical.c:126-214) */
typedef struct {
  int* head;
  int* next;
  int* prev;
} buckets;

static void bk_remove(buckets* b, int x, int key) {
  if (b->prev[x] >= 0) b->next[b->prev[x]] = b->next[x];
  else b->head[key] = b->next[x];
  if (b->next[x] >= 0) b->prev[b->next[x]] = b->prev[x];
}
static void bk_push(buckets* b, int x, int key) {
  b->next[x] = b->head[key];
  b->prev[x] = -1;
  if (b->head[key] >= 0) b->prev[b->head[key]] = x;
  b->head[key] = x;
}

/* Greedy first pass shared by RS and HMIS.  `limit_processed` reproduces the
 * HMIS loop guard (rs_classical.c:441), which stops after n decisions. */
static void rs_greedy(const orc_csr* s, const orc_csr* st, int* lambda, int nb, int top,
                      int* cf, int limit_processed) {
  const int n = s->n;
  buckets b;
  b.head = (int*)xcalloc((size_t)nb, sizeof(int));
  b.next = (int*)xcalloc((size_t)n, sizeof(int));
  b.prev = (int*)xcalloc((size_t)n, sizeof(int));
  for (int k = 0; k < nb; k++) b.head[k] = -1;
  for (int i = n - 1; i >= 0; i--) bk_push(&b, i, lambda[i]);
  int processed = 0;
  for (;;) {
    if (limit_processed && processed >= n) break;
    while (top >= 0 && b.head[top] < 0) top--;
    if (top < 0) break;
    const int best = b.head[top];
    bk_remove(&b, best, lambda[best]);
    cf[best] = C_PT;
    processed++;
    for (int q = st->ia[best]; q < st->ia[best + 1]; q++) {
      const int j = st->ja[q];
      if (cf[j] != UNDEC) continue;
      bk_remove(&b, j, lambda[j]);
      cf[j] = F_PT;
      processed++;
      for (int r = s->ia[j]; r < s->ia[j + 1]; r++) {
        const int k = s->ja[r];
        if (cf[k] != UNDEC) continue;
        bk_remove(&b, k, lambda[k]);
        lambda[k]++;
        bk_push(&b, k, lambda[k]);
        if (lambda[k] > top) top = lambda[k];
      }
    }
  }
  free(b.head);
  free(b.next);
  free(b.prev);
}

/* F points without a strong C neighbour become C, scanning i = 0..n-1 and
 * updating in place (rs_classical.c:214-221, :357-364, :595-602). */
static int second_pass(const orc_csr* s, int* cf) {
  const int n = s->n;
  for (int i = 0; i < n; i++) {
    if (cf[i] != F_PT) continue;
    int has_c = 0;
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++)
      if (cf[s->ja[k]] == C_PT) { has_c = 1; break; }
    if (!has_c) cf[i] = C_PT;
  }
  int nc = 0;
  for (int i = 0; i < n; i++) nc += (cf[i] == C_PT);
  return nc;
}

/* Classical RS: rs_classical.c:108-229 (lambda[0] is left at zero). */
void orc_rs(const orc_csr* s, int max_lam, int* cf, int* nc) {
  const int n = s->n;
  orc_csr st;
  orc_transpose(s, &st);
  int* lambda = (int*)xcalloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++) cf[i] = UNDEC;
  for (int i = 1; i < n; i++) lambda[i] = st.ia[i + 1] - st.ia[i];
  /* the reference sizes 2*max_lam+1 buckets; more are kept here so a
   * measure that outgrows them stays defined */
  int nb = 2 * max_lam + 1;
  int need = n + max_lam + 2;
  if (nb < need) nb = need;
  rs_greedy(s, &st, lambda, nb, max_lam, cf, 0);
  *nc = second_pass(s, cf);
  free(lambda);
  orc_csr_free(&st);
}

/* G = S u S^T without the diagonal, S entries first (rs_classical.c:262-290) */
static void build_g(const orc_csr* s, const orc_csr* st, int** gia, int** gja) {
  const int n = s->n;
  int* mark = (int*)xcalloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++) mark[i] = -1;
  int* ia = (int*)xcalloc((size_t)n + 1, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    int* ja = pass ? (int*)xcalloc((size_t)ia[n], sizeof(int)) : NULL;
    for (int i = 0; i < n; i++) mark[i] = -1;
    for (int i = 0; i < n; i++) {
      int c = pass ? ia[i] : 0;
      for (int k = s->ia[i]; k < s->ia[i + 1]; k++) {
        int j = s->ja[k];
        if (j != i && mark[j] != i) { mark[j] = i; if (pass) ja[c] = j; c++; }
      }
      for (int k = st->ia[i]; k < st->ia[i + 1]; k++) {
        int j = st->ja[k];
        if (j != i && mark[j] != i) { mark[j] = i; if (pass) ja[c] = j; c++; }
      }
      if (!pass) ia[i + 1] = c;
    }
    if (!pass)
      for (int i = 0; i < n; i++) ia[i + 1] += ia[i];
    else
      *gja = ja;
  }
  *gia = ia;
  free(mark);
}

/* Jacobi-style independent-set rounds (rs_classical.c:305-350). */
static void pmis_rounds(int n, const int* gia, const int* gja, const double* w, int* cf,
                        int undecided) {
  int* newc = (int*)xcalloc((size_t)n, sizeof(int));
  while (undecided > 0) {
    int m = 0;
    for (int i = 0; i < n; i++) {
      if (cf[i] != UNDEC) continue;
      int best = 1;
      for (int k = gia[i]; k < gia[i + 1]; k++) {
        int j = gja[k];
        if (cf[j] == UNDEC && w[j] > w[i]) { best = 0; break; }
      }
      if (best) newc[m++] = i;
    }
    if (m == 0) {
      for (int i = 0; i < n; i++)
        if (cf[i] == UNDEC) { cf[i] = C_PT; undecided--; }
      break;
    }
    for (int q = 0; q < m; q++) { cf[newc[q]] = C_PT; undecided--; }
    for (int i = 0; i < n; i++) {
      if (cf[i] != UNDEC) continue;
      for (int k = gia[i]; k < gia[i + 1]; k++)
        if (cf[gja[k]] == C_PT) { cf[i] = F_PT; undecided--; break; }
    }
  }
  free(newc);
}

/* PMIS: rs_classical.c:246-371. */
void orc_pmis(const orc_csr* s, int* cf, int* nc) {
  const int n = s->n;
  orc_csr st;
  orc_transpose(s, &st);
  int *gia, *gja;
  build_g(s, &st, &gia, &gja);
  double* w = (double*)xcalloc((size_t)n, sizeof(double));
  srand(12345);
  for (int i = 0; i < n; i++) {
    int lam = st.ia[i + 1] - st.ia[i];
    w[i] = (double)lam + (double)rand() / (double)RAND_MAX;
    cf[i] = UNDEC;
  }
  pmis_rounds(n, gia, gja, w, cf, n);
  *nc = second_pass(s, cf);
  free(w);
  free(gia);
  free(gja);
  orc_csr_free(&st);
}

/* HMIS: greedy first pass, then PMIS on what is left (rs_classical.c:390-611). */
void orc_hmis(const orc_csr* s, int* cf, int* nc) {
  const int n = s->n;
  orc_csr st;
  orc_transpose(s, &st);
  int* lambda = (int*)xcalloc((size_t)n, sizeof(int));
  int maxl = 0, maxrow = 0;
  for (int i = 0; i < n; i++) {
    lambda[i] = st.ia[i + 1] - st.ia[i];
    cf[i] = UNDEC;
    if (lambda[i] > maxl) maxl = lambda[i];
    int rl = s->ia[i + 1] - s->ia[i];
    if (rl > maxrow) maxrow = rl;
  }
  int nb = maxl + maxrow + 1;
  int need = n + maxl + 2;
  if (nb < need) nb = need;
  rs_greedy(s, &st, lambda, nb, maxl, cf, 1);
  int undecided = 0;
  for (int i = 0; i < n; i++) undecided += (cf[i] == UNDEC);
  if (undecided > 0) {
    int *gia, *gja;
    build_g(s, &st, &gia, &gja);
    double* w = (double*)xcalloc((size_t)n, sizeof(double));
    srand(12345);
    for (int i = 0; i < n; i++)
      w[i] = (cf[i] == UNDEC)
                 ? (double)(st.ia[i + 1] - st.ia[i]) + (double)rand() / (double)RAND_MAX
                 : -1.0;
    pmis_rounds(n, gia, gja, w, cf, undecided);
    free(w);
    free(gia);
    free(gja);
  }
  *nc = second_pass(s, cf);
  free(lambda);
  orc_csr_free(&st);
}

/* Direct interpolation, pattern and values: rs_classical.c:643-805. */
void orc_interp(const orc_csr* a, const orc_csr* s, const int* cf, orc_csr* p) {
  const int n = a->n;
  int* cmap = (int*)xcalloc((size_t)n, sizeof(int));
  int nc = 0;
  for (int i = 0; i < n; i++) cmap[i] = (cf[i] == C_PT) ? nc++ : -1;
  int total = 0;
  for (int i = 0; i < n; i++) {
    if (cf[i] == C_PT) { total++; continue; }
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++) total += (cf[s->ja[k]] == C_PT);
  }
  csr_alloc(p, n, nc, total);
  int q = 0;
  for (int i = 0; i < n; i++) {
    p->ia[i] = q;
    if (cf[i] == C_PT) { p->ja[q++] = cmap[i]; continue; }
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++)
      if (cf[s->ja[k]] == C_PT) p->ja[q++] = cmap[s->ja[k]];
  }
  p->ia[n] = q;
  /* values */
  int* strong_of = (int*)xcalloc((size_t)n, sizeof(int));
  int* slot = (int*)xcalloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++) { strong_of[i] = -1; slot[i] = -1; }
  for (int i = 0; i < n; i++) {
    if (cf[i] == C_PT) { p->val[p->ia[i]] = 1.0; continue; }
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++) strong_of[s->ja[k]] = i;
    int r = p->ia[i];
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++) {
      int j = s->ja[k];
      if (cf[j] == C_PT) { p->val[r] = 0.0; slot[j] = r; r++; }
    }
    double diag = 0.0, weak = 0.0;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      int j = a->ja[k];
      double v = a->val[k];
      if (j == i) diag = v;
      else if (strong_of[j] == i && cf[j] == C_PT) p->val[slot[j]] += v;
      else if (strong_of[j] == i && cf[j] == F_PT) { /* below */ }
      else weak += v;
    }
    double dh = diag + weak;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
      int kk = a->ja[k];
      if (kk == i || strong_of[kk] != i || cf[kk] != F_PT) continue;
      double aik = a->val[k];
      double den = 0.0;
      for (int l = a->ia[kk]; l < a->ia[kk + 1]; l++) {
        int mcol = a->ja[l];
        if (cf[mcol] == C_PT && strong_of[mcol] == i) den += a->val[l];
      }
      if (fabs(den) < 1e-15) {
        dh += aik;
      } else {
        for (int l = a->ia[kk]; l < a->ia[kk + 1]; l++) {
          int mcol = a->ja[l];
          if (cf[mcol] == C_PT && strong_of[mcol] == i) p->val[slot[mcol]] += aik * a->val[l] / den;
        }
      }
    }
    if (fabs(dh) > 1e-15)
      for (int r2 = p->ia[i]; r2 < p->ia[i + 1]; r2++) p->val[r2] /= -dh;
    for (int k = s->ia[i]; k < s->ia[i + 1]; k++)
      if (cf[s->ja[k]] == C_PT) slot[s->ja[k]] = -1;
  }
  free(cmap);
  free(strong_of);
  free(slot);
}

/* Galerkin triple product, diagonal first then discovery order:
 * sparse_ops.c:102-213. */
void orc_rap(const orc_csr* r, const orc_csr* a, const orc_csr* p, orc_csr* ac) {
  const int nc = r->n, nf = a->n;
  int* where = (int*)xcalloc((size_t)p->m, sizeof(int));  /* column -> output slot */
  int* seen = (int*)xcalloc((size_t)nf, sizeof(int));
  for (int j = 0; j < p->m; j++) where[j] = -1;
  for (int j = 0; j < nf; j++) seen[j] = -1;
  int* ia = (int*)xcalloc((size_t)nc + 1, sizeof(int));
  int cnt = 0;
  for (int ic = 0; ic < nc; ic++) {
    const int row0 = cnt;
    where[ic] = cnt++;
    for (int k1 = r->ia[ic]; k1 < r->ia[ic + 1]; k1++) {
      int i1 = r->ja[k1];
      for (int k2 = a->ia[i1]; k2 < a->ia[i1 + 1]; k2++) {
        int i2 = a->ja[k2];
        if (seen[i2] == ic) continue;
        seen[i2] = ic;
        for (int k3 = p->ia[i2]; k3 < p->ia[i2 + 1]; k3++)
          if (where[p->ja[k3]] < row0) where[p->ja[k3]] = cnt++;
      }
    }
    ia[ic] = row0;
  }
  ia[nc] = cnt;
  ac->n = nc;
  ac->m = p->m;
  ac->nnz = cnt;
  ac->ia = ia;
  ac->ja = (int*)xcalloc((size_t)cnt, sizeof(int));
  ac->val = (double*)xcalloc((size_t)cnt, sizeof(double));
  for (int j = 0; j < p->m; j++) where[j] = -1;
  for (int j = 0; j < nf; j++) seen[j] = -1;
  int pos = 0;
  for (int ic = 0; ic < nc; ic++) {
    const int row0 = pos;
    where[ic] = pos;
    ac->ja[pos] = ic;
    ac->val[pos] = 0.0;
    pos++;
    for (int k1 = r->ia[ic]; k1 < r->ia[ic + 1]; k1++) {
      double rv = r->val[k1];
      int i1 = r->ja[k1];
      for (int k2 = a->ia[i1]; k2 < a->ia[i1 + 1]; k2++) {
        double ra = rv * a->val[k2];
        int i2 = a->ja[k2];
        seen[i2] = ic;
        for (int k3 = p->ia[i2]; k3 < p->ia[i2 + 1]; k3++) {
          double v = ra * p->val[k3];
          int i3 = p->ja[k3];
          if (where[i3] < row0) {
            where[i3] = pos;
            ac->ja[pos] = i3;
            ac->val[pos] = v;
            pos++;
          } else {
            ac->val[where[i3]] += v;
          }
        }
      }
    }
  }
  free(where);
  free(seen);
}

/* IC(0) on the lower triangle: ichol.c:12-118. */
void orc_ichol(const orc_csr* a, orc_csr* l) {
  const int n = a->n;
  int cnt = 0;
  for (int i = 0; i < n; i++)
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) cnt += (a->ja[k] <= i);
  csr_alloc(l, n, n, cnt);
  int p = 0;
  for (int i = 0; i < n; i++) {
    l->ia[i] = p;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++)
      if (a->ja[k] <= i) {
        l->ja[p] = a->ja[k];
        l->val[p] = a->val[k];
        p++;
      }
  }
  l->ia[n] = p;
  double* w = (double*)xcalloc((size_t)n, sizeof(double));
  int* owner = (int*)xcalloc((size_t)n, sizeof(int));
  int* dpos = (int*)xcalloc((size_t)n, sizeof(int));
  for (int i = 0; i < n; i++) {
    owner[i] = -1;
    dpos[i] = -1;
    for (int k = l->ia[i]; k < l->ia[i + 1]; k++)
      if (l->ja[k] == i) { dpos[i] = k; break; }
  }
  for (int i = 0; i < n; i++) {
    for (int k = l->ia[i]; k < l->ia[i + 1]; k++) {
      w[l->ja[k]] = l->val[k];
      owner[l->ja[k]] = i;
    }
    for (int kk = l->ia[i]; kk < l->ia[i + 1]; kk++) {
      int k = l->ja[kk];
      if (k >= i) continue;
      double s = w[k];
      for (int jj = l->ia[k]; jj < l->ia[k + 1]; jj++) {
        int j = l->ja[jj];
        if (j >= k) break;
        if (owner[j] == i) s -= w[j] * l->val[jj];
      }
      w[k] = s / l->val[dpos[k]];
    }
    double d = w[i];
    for (int kk = l->ia[i]; kk < l->ia[i + 1]; kk++) {
      int j = l->ja[kk];
      if (j >= i) break;
      d -= w[j] * w[j];
    }
    if (d <= 0.0) d = 1e-14;
    w[i] = sqrt(d);
    for (int kk = l->ia[i]; kk < l->ia[i + 1]; kk++) l->val[kk] = w[l->ja[kk]];
    for (int kk = l->ia[i]; kk < l->ia[i + 1]; kk++) {
      w[l->ja[kk]] = 0.0;
      owner[l->ja[kk]] = -1;
    }
  }
  free(w);
  free(owner);
  free(dpos);
}

/* L L^T x = b: ichol.c:121-165 (column-oriented backward sweep). */
void orc_ichol_solve(const orc_csr* l, const double* b, double* x) {
  const int n = l->n;
  double* y = (double*)xcalloc((size_t)n, sizeof(double));
  for (int i = 0; i < n; i++) {
    double s = b[i], d = 1.0;
    for (int k = l->ia[i]; k < l->ia[i + 1]; k++) {
      int j = l->ja[k];
      if (j < i) s -= l->val[k] * y[j];
      else if (j == i) d = l->val[k];
    }
    y[i] = s / d;
  }
  memcpy(x, y, sizeof(double) * (size_t)n);
  double* dg = (double*)xcalloc((size_t)n, sizeof(double));
  for (int i = 0; i < n; i++)
    for (int k = l->ia[i]; k < l->ia[i + 1]; k++)
      if (l->ja[k] == i) { dg[i] = l->val[k]; break; }
  for (int i = n - 1; i >= 0; i--) {
    x[i] /= dg[i];
    for (int k = l->ia[i]; k < l->ia[i + 1]; k++) {
      int j = l->ja[k];
      if (j < i) x[j] -= l->val[k] * x[i];
    }
  }
  free(y);
  free(dg);
}

/* SpMV family: sparse_ops.c:19-75. */
void orc_spmv(const orc_csr* a, const double* x, double* y) {
  for (int i = 0; i < a->n; i++) {
    double h = 0.0;
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) h += a->val[k] * x[a->ja[k]];
    y[i] = h;
  }
}
void orc_residual(const orc_csr* a, const double* b, const double* x, double* r) {
  for (int i = 0; i < a->n; i++) {
    double h = b[i];
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) h -= a->val[k] * x[a->ja[k]];
    r[i] = h;
  }
}
void orc_spmv_add(const orc_csr* a, const double* x, double* y) {
  for (int i = 0; i < a->n; i++) {
    double h = y[i];
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) h += a->val[k] * x[a->ja[k]];
    y[i] = h;
  }
}
void orc_spmv_t(const orc_csr* a, const double* x, int m, double* y) {
  for (int j = 0; j < m; j++) y[j] = 0.0;
  for (int i = 0; i < a->n; i++) {
    double h = x[i];
    for (int k = a->ia[i]; k < a->ia[i + 1]; k++) y[a->ja[k]] += a->val[k] * h;
  }
}

/* ------------------------------------------------------------------ solver */
#define MAXLEV 20

typedef struct {
  orc_csr A, S, P;
  int* cf;
  int* order;  /* C points then F points (build_hierarchy.c:92-97) */
  double* l1;
  int n, nc;
} orc_level;

typedef struct {
  orc_csr A;          /* solve matrix */
  orc_level lv[MAXLEV];
  int nlev;
  orc_csr Lc;         /* coarsest ichol */
  orc_csr L;          /* fine ichol */
  int nu, smoother;
  double omega;
} orc_solver;

static double dot(const double* u, const double* v, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += u[i] * v[i];
  return s;
}

typedef void (*precond_fn)(const void*, const double*, double*);

/* PCG with a preconditioner callback: amg_pcg.c:12-101. */
static int pcg(const orc_csr* a, const double* b, double* x, precond_fn pre, const void* pd,
               double tol, int maxiter) {
  const int n = a->n;
  double* r = (double*)xcalloc((size_t)n, sizeof(double));
  double* z = (double*)xcalloc((size_t)n, sizeof(double));
  double* p = (double*)xcalloc((size_t)n, sizeof(double));
  double* ap = (double*)xcalloc((size_t)n, sizeof(double));
  orc_residual(a, b, x, r);
  pre(pd, r, z);
  memcpy(p, z, sizeof(double) * (size_t)n);
  double rz = dot(r, z, n);
  const double rz0 = rz;
  int it;
  for (it = 1; it <= maxiter; it++) {
    orc_spmv(a, p, ap);
    double pap = dot(p, ap, n);
    double alpha = rz / pap;
    for (int i = 0; i < n; i++) x[i] = x[i] + p[i] * alpha;
    for (int i = 0; i < n; i++) r[i] = r[i] + ap[i] * (-alpha);
    pre(pd, r, z);
    double rzn = dot(r, z, n);
    if (sqrt(rzn / rz0) < tol) break;
    double beta = rzn / rz;
    rz = rzn;
    for (int i = 0; i < n; i++) p[i] = beta * p[i] + z[i];
  }
  if (it > maxiter) it = -maxiter;
  free(r);
  free(z);
  free(p);
  free(ap);
  return it;
}

static void ichol_pre(const void* d, const double* g, double* x) {
  orc_ichol_solve((const orc_csr*)d, g, x);
}

/* one row of Gauss-Seidel, diagonal fallback 1.0 (amg_cycle.c:21-80) */
static void gs_row(const orc_csr* a, int i, const double* b, double* x) {
  double s = b[i], d = 1.0;
  for (int k = a->ia[i]; k < a->ia[i + 1]; k++) {
    if (a->ja[k] == i) d = a->val[k];
    else s -= a->val[k] * x[a->ja[k]];
  }
  x[i] = s / d;
}

/* smoother dispatch (amg_cycle.c:137-175) */
static void smooth(const orc_solver* S, int l, const double* b, double* x, int forward) {
  const orc_level* L = &S->lv[l];
  const int n = L->n;
  for (int sw = 0; sw < S->nu; sw++) {
    if (S->smoother == 2 || S->smoother == 1) {
      for (int q = 0; q < n; q++) {
        int ii = forward ? q : n - 1 - q;
        gs_row(&L->A, S->smoother == 2 ? L->order[ii] : ii, b, x);
      }
    } else {
      double* r = (double*)xcalloc((size_t)n, sizeof(double));
      for (int i = 0; i < n; i++) {
        double s = b[i], d = 1.0;
        for (int k = L->A.ia[i]; k < L->A.ia[i + 1]; k++) {
          if (S->smoother == 3 && L->A.ja[k] == i) d = L->A.val[k];
          s -= L->A.val[k] * x[L->A.ja[k]];
        }
        r[i] = (S->smoother == 3) ? s / d : s;
      }
      for (int i = 0; i < n; i++) x[i] += (S->smoother == 3) ? S->omega * r[i] : r[i] / L->l1[i];
      free(r);
    }
  }
}

/* backslash_rec / fwdslash_rec (amg_cycle.c:180-253) */
static void cycle(const orc_solver* S, int l, const double* b, double* x, int back) {
  const orc_level* L = &S->lv[l];
  if (l == S->nlev - 1) {
    pcg(&L->A, b, x, ichol_pre, &S->Lc, 1e-12, L->n);
    return;
  }
  const int n = L->n, nc = L->nc;
  if (back) smooth(S, l, b, x, 1);
  double* r = (double*)xcalloc((size_t)n, sizeof(double));
  double* rc = (double*)xcalloc((size_t)nc, sizeof(double));
  double* ec = (double*)xcalloc((size_t)nc, sizeof(double));
  orc_residual(&L->A, b, x, r);
  orc_spmv_t(&L->P, r, nc, rc);
  cycle(S, l + 1, rc, ec, back);
  orc_spmv_add(&L->P, ec, x);
  if (!back) smooth(S, l, b, x, 0);
  free(r);
  free(rc);
  free(ec);
}

/* three-stage AMG + IC(0) preconditioner (amg_ichol_precond.c:22-48) */
void orc_precond(void* h, const double* g, double* x) {
  const orc_solver* S = (const orc_solver*)h;
  const int n = S->A.n;
  double* u1 = (double*)xcalloc((size_t)n, sizeof(double));
  double* r1 = (double*)xcalloc((size_t)n, sizeof(double));
  double* ic = (double*)xcalloc((size_t)n, sizeof(double));
  double* r2 = (double*)xcalloc((size_t)n, sizeof(double));
  double* co = (double*)xcalloc((size_t)n, sizeof(double));
  cycle(S, 0, g, u1, 1);
  orc_residual(&S->A, g, u1, r1);
  orc_ichol_solve(&S->L, r1, ic);
  for (int i = 0; i < n; i++) x[i] = u1[i];
  for (int i = 0; i < n; i++) x[i] = x[i] + ic[i] * 1.0;
  orc_residual(&S->A, g, x, r2);
  cycle(S, 0, r2, co, 0);
  for (int i = 0; i < n; i++) x[i] = x[i] + co[i] * 1.0;
  free(u1);
  free(r1);
  free(ic);
  free(r2);
  free(co);
}

static void precond_cb(const void* d, const double* g, double* x) { orc_precond((void*)d, g, x); }

/* amg_solver_create (amg_wrapper.c:51-97) + amg_build_hierarchy
 * (build_hierarchy.c:29-156) with a selectable coarsening. */
void* orc_create(int n, int nnz, const int* ia, const int* ja, const double* val,
                 double theta, int min_size, int max_levels, int nu, int coarsening,
                 int smoother, double omega) {
  orc_solver* S = (orc_solver*)xcalloc(1, sizeof(orc_solver));
  orc_csr in;
  csr_alloc(&in, n, n, nnz);
  memcpy(in.ia, ia, sizeof(int) * ((size_t)n + 1));
  memcpy(in.ja, ja, sizeof(int) * (size_t)nnz);
  memcpy(in.val, val, sizeof(double) * (size_t)nnz);
  orc_symmetrize(&in, &S->A);
  orc_csr_free(&in);
  S->nu = nu > 0 ? nu : 1;
  S->smoother = smoother;
  S->omega = omega;
  if (max_levels <= 0 || max_levels > MAXLEV) max_levels = MAXLEV;
  /* level 0 holds a copy of A */
  orc_level* L0 = &S->lv[0];
  csr_alloc(&L0->A, n, n, S->A.nnz);
  memcpy(L0->A.ia, S->A.ia, sizeof(int) * ((size_t)n + 1));
  memcpy(L0->A.ja, S->A.ja, sizeof(int) * (size_t)S->A.nnz);
  memcpy(L0->A.val, S->A.val, sizeof(double) * (size_t)S->A.nnz);
  L0->n = n;
  int nlev = 1;
  while (S->lv[nlev - 1].A.n >= min_size && nlev < max_levels) {
    orc_level* cur = &S->lv[nlev - 1];
    const int nf = cur->A.n;
    int ml = 0, nc = 0;
    orc_strength(&cur->A, theta, &cur->S, &ml);
    int* cf = (int*)xcalloc((size_t)nf, sizeof(int));
    if (coarsening == 1) orc_pmis(&cur->S, cf, &nc);
    else if (coarsening == 2) orc_hmis(&cur->S, cf, &nc);
    else orc_rs(&cur->S, ml, cf, &nc);
    cur->nc = nc;
    if (nc == 0 || nc >= nf) { free(cf); break; }
    cur->cf = cf;
    cur->order = (int*)xcalloc((size_t)nf, sizeof(int));
    int q = 0;
    for (int i = 0; i < nf; i++) if (cf[i] == C_PT) cur->order[q++] = i;
    for (int i = 0; i < nf; i++) if (cf[i] != C_PT) cur->order[q++] = i;
    orc_interp(&cur->A, &cur->S, cf, &cur->P);
    orc_csr pt, ac;
    orc_transpose(&cur->P, &pt);
    orc_rap(&pt, &cur->A, &cur->P, &ac);
    orc_csr_free(&pt);
    orc_level* nx = &S->lv[nlev];
    orc_symmetrize(&ac, &nx->A);
    orc_csr_free(&ac);
    nx->n = nc;
    nlev++;
  }
  S->nlev = nlev;
  for (int l = 0; l < nlev; l++) {
    orc_level* L = &S->lv[l];
    L->l1 = (double*)xcalloc((size_t)L->A.n, sizeof(double));
    for (int i = 0; i < L->A.n; i++) {
      double s = 0.0;
      for (int k = L->A.ia[i]; k < L->A.ia[i + 1]; k++) s += fabs(L->A.val[k]);
      L->l1[i] = s;
    }
  }
  orc_ichol(&S->lv[nlev - 1].A, &S->Lc);
  orc_ichol(&S->A, &S->L);
  return S;
}

int orc_solve(void* h, const double* b, double* x, double tol, int maxiter) {
  orc_solver* S = (orc_solver*)h;
  return pcg(&S->A, b, x, precond_cb, S, tol, maxiter);
}

int orc_num_levels(void* h) { return ((orc_solver*)h)->nlev; }

void orc_level_sizes(void* h, int k, int* o) {
  orc_solver* S = (orc_solver*)h;
  orc_level* L = &S->lv[k];
  int last = (k == S->nlev - 1);
  o[0] = L->A.n;
  o[1] = L->A.nnz;
  o[2] = last ? 0 : L->S.nnz;
  o[3] = last ? 0 : L->P.nnz;
  o[4] = last ? 0 : L->nc;
}

void orc_level_copy(void* h, int k, int* a_ia, int* a_ja, double* a_val, int* s_ia,
                    int* s_ja, double* s_val, int* p_ia, int* p_ja, double* p_val, int* cf) {
  orc_solver* S = (orc_solver*)h;
  orc_level* L = &S->lv[k];
  const int n = L->A.n;
  memcpy(a_ia, L->A.ia, sizeof(int) * ((size_t)n + 1));
  memcpy(a_ja, L->A.ja, sizeof(int) * (size_t)L->A.nnz);
  memcpy(a_val, L->A.val, sizeof(double) * (size_t)L->A.nnz);
  if (k == S->nlev - 1) return;
  memcpy(s_ia, L->S.ia, sizeof(int) * ((size_t)n + 1));
  memcpy(s_ja, L->S.ja, sizeof(int) * (size_t)L->S.nnz);
  memcpy(s_val, L->S.val, sizeof(double) * (size_t)L->S.nnz);
  memcpy(p_ia, L->P.ia, sizeof(int) * ((size_t)n + 1));
  memcpy(p_ja, L->P.ja, sizeof(int) * (size_t)L->P.nnz);
  memcpy(p_val, L->P.val, sizeof(double) * (size_t)L->P.nnz);
  memcpy(cf, L->cf, sizeof(int) * (size_t)n);
}

int orc_ichol_nnz(void* h) { return ((orc_solver*)h)->L.nnz; }
void orc_ichol_copy(void* h, int* ia, int* ja, double* val) {
  orc_solver* S = (orc_solver*)h;
  memcpy(ia, S->L.ia, sizeof(int) * ((size_t)S->L.n + 1));
  memcpy(ja, S->L.ja, sizeof(int) * (size_t)S->L.nnz);
  memcpy(val, S->L.val, sizeof(double) * (size_t)S->L.nnz);
}

void orc_free(void* h) {
  orc_solver* S = (orc_solver*)h;
  if (!S) return;
  orc_csr_free(&S->A);
  orc_csr_free(&S->L);
  orc_csr_free(&S->Lc);
  for (int l = 0; l < S->nlev; l++) {
    orc_level* L = &S->lv[l];
    orc_csr_free(&L->A);
    orc_csr_free(&L->S);
    orc_csr_free(&L->P);
    free(L->cf);
    free(L->order);
    free(L->l1);
  }
  free(S);
}
