/*
 * CPU restatement of the reference's Hamiltonian path (see mcd_oracle.h).
 * TEST INFRASTRUCTURE ONLY.
 */
#include "mcd_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXW 2

typedef struct {
  int a, b;
  double v;
} dentry;

typedef struct {
  int a;
  double h;
  double* t; /* [nso] */
} sentry;

struct oracle {
  int nso, nelec, ms2, uhf, nw;
  double ecore;
  double thr;
  double* h1;
  double* g;
  unsigned char* gset;
  int n_oe;
  int* oe_idx;
  double* oe_val;
  dentry** dbl;
  int* ndbl;
  sentry** sgl;
  int* nsgl;
  double* d1;
  double* d2;
};

static size_t gidx(const oracle* o, int i, int j, int a, int b) {
  const size_t n = (size_t)o->nso;
  return (((size_t)i * n + j) * n + a) * n + b;
}

/* src/input.h:319-330: 0 when the key is absent (only keys i <= j exist). */
static double G(const oracle* o, int i, int j, int a, int b) {
  if (i > j) return 0.0;
  return o->g[gidx(o, i, j, a, b)];
}

static void put(oracle* o, int i, int j, int a, int b, double v) {
  const size_t x = gidx(o, i, j, a, b);
  if (!o->gset[x]) {
    o->g[x] = v;
    o->gset[x] = 1;
  }
}

/* insert_two_body_ (src/input.h:304-316). */
static void ins(oracle* o, int i, int j, int a, int b, double v) {
  if (i <= j) put(o, i, j, a, b, v);
  if (i >= j) put(o, j, i, b, a, v);
}

static void rhf_ins(oracle* o, int i, int j, int a, int b, double v) {
  ins(o, 2 * i - 2, 2 * j - 2, 2 * a - 2, 2 * b - 2, v);
  ins(o, 2 * i - 1, 2 * j - 1, 2 * a - 1, 2 * b - 1, v);
  ins(o, 2 * i - 2, 2 * j - 1, 2 * a - 2, 2 * b - 1, v);
  ins(o, 2 * i - 1, 2 * j - 2, 2 * a - 1, 2 * b - 2, v);
}

static void add_oe(oracle* o, int i, double v) {
  for (int x = 0; x < o->n_oe; ++x)
    if (o->oe_idx[x] == i) return; /* first insertion wins */
  o->oe_idx[o->n_oe] = i;
  o->oe_val[o->n_oe] = v;
  o->n_oe++;
}

static int find_int(const char* hdr, const char* name, int* out) {
  const char* p = hdr;
  size_t nl = strlen(name);
  while ((p = strstr(p, name)) != NULL) {
    const char* q = p + nl;
    while (*q == ' ') ++q;
    if (*q == '=') {
      ++q;
      while (*q == ' ') ++q;
      if (*q >= '0' && *q <= '9') {
        *out = atoi(q);
        return 1;
      }
    }
    p += nl;
  }
  return 0;
}

static int find_uhf(const char* hdr) {
  const char* p = hdr;
  while ((p = strstr(p, "UHF")) != NULL) {
    const char* q = p + 3;
    while (*q == ' ') ++q;
    if (*q == '=') {
      ++q;
      while (*q == ' ' || *q == '.') ++q;
      if (strncmp(q, "TRUE", 4) == 0) return 1;
      if (strncmp(q, "FALSE", 5) == 0) return 0;
    }
    p += 3;
  }
  return 0;
}

static int cmp_dentry(const void* x, const void* y) {
  const double a = fabs(((const dentry*)x)->v), b = fabs(((const dentry*)y)->v);
  return (a < b) - (a > b);
}

static int cmp_sentry(const void* x, const void* y) {
  const double a = fabs(((const sentry*)x)->h), b = fabs(((const sentry*)y)->h);
  return (a < b) - (a > b);
}

/* construct_double_excitation (src/hamiltonian.h:113-173). */
static void build_doubles(oracle* o) {
  const int n = o->nso;
  o->dbl = calloc((size_t)n * n, sizeof(dentry*));
  o->ndbl = calloc((size_t)n * n, sizeof(int));
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      int cap = 64, cnt = 0;
      dentry* L = malloc(cap * sizeof(dentry));
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
          const size_t x = gidx(o, i, j, a, b);
          if (!o->gset[x]) continue;
          const double v = o->g[x];
          dentry e;
          int keep = 0;
          if ((i % 2) ^ (j % 2)) {
            if (fabs(v) > o->thr) {
              e.a = a;
              e.b = b;
              e.v = v;
              keep = 1;
            }
          } else if (a < b) {
            const double w = v - G(o, i, j, b, a);
            if (fabs(w) > o->thr) {
              e.a = a;
              e.b = b;
              e.v = w;
              keep = 1;
            }
          } else if (b < a && !o->gset[gidx(o, i, j, b, a)]) {
            const double w = -v;
            if (fabs(w) > o->thr) {
              e.a = b;
              e.b = a;
              e.v = w;
              keep = 1;
            }
          }
          if (keep) {
            if (cnt == cap) {
              cap *= 2;
              L = realloc(L, cap * sizeof(dentry));
            }
            L[cnt++] = e;
          }
        }
      qsort(L, cnt, sizeof(dentry), cmp_dentry);
      o->dbl[i * n + j] = L;
      o->ndbl[i * n + j] = cnt;
    }
}

/* construct_single_excitation (src/hamiltonian.h:176-219). */
static void build_singles(oracle* o) {
  const int n = o->nso;
  o->sgl = calloc(n, sizeof(sentry*));
  o->nsgl = calloc(n, sizeof(int));
  for (int i = 0; i < n; ++i) {
    sentry* L = malloc((size_t)n * sizeof(sentry));
    int cnt = 0;
    for (int a = 0; a < n; ++a) {
      sentry e;
      e.a = a;
      e.h = o->h1[i * n + a];
      e.t = malloc((size_t)n * sizeof(double));
      double mx = fabs(e.h);
      for (int k = 0; k < n; ++k) {
        double v;
        if (i <= k)
          v = G(o, i, k, a, k) - G(o, i, k, k, a);
        else
          v = G(o, k, i, k, a) - G(o, k, i, a, k);
        e.t[k] = v;
        if (fabs(v) > mx) mx = fabs(v);
      }
      if (mx > o->thr)
        L[cnt++] = e;
      else
        free(e.t);
    }
    qsort(L, cnt, sizeof(sentry), cmp_sentry);
    o->sgl[i] = L;
    o->nsgl[i] = cnt;
  }
}

static void build_diagonal(oracle* o) {
  const int n = o->nso;
  o->d1 = calloc(n, sizeof(double));
  o->d2 = calloc((size_t)n * n, sizeof(double));
  for (int i = 0; i < n; ++i) o->d1[i] = o->h1[i * n + i];
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) o->d2[i * n + j] = G(o, i, j, i, j) - G(o, i, j, j, i);
}

oracle* oracle_load(const char* path, double thr, char* err, int errlen) {
  FILE* f = fopen(path, "r");
  if (!f) {
    snprintf(err, errlen, "cannot open %s", path);
    return NULL;
  }
  char line[4096];
  size_t hcap = 1 << 16, hlen = 0;
  char* hdr = calloc(hcap, 1);
  int ended = 0;
  while (fgets(line, sizeof line, f)) {
    if (strstr(line, "&END") || strchr(line, '/')) {
      ended = 1;
      break;
    }
    size_t l = strlen(line);
    if (hlen + l + 2 >= hcap) {
      hcap *= 2;
      hdr = realloc(hdr, hcap);
    }
    hdr[hlen++] = ' ';
    memcpy(hdr + hlen, line, l);
    hlen += l;
    hdr[hlen] = 0;
  }
  if (!ended) {
    snprintf(err, errlen, "FCIDUMP has the wrong header.");
    fclose(f);
    free(hdr);
    return NULL;
  }
  oracle* o = calloc(1, sizeof(oracle));
  int norb = 0;
  if (!find_int(hdr, "NORB", &norb) || !find_int(hdr, "NELEC", &o->nelec) || !find_int(hdr, "MS2", &o->ms2)) {
    snprintf(err, errlen, "header parameter missing");
    fclose(f);
    free(hdr);
    free(o);
    return NULL;
  }
  o->uhf = find_uhf(hdr);
  free(hdr);
  o->nso = o->uhf ? norb : 2 * norb;
  o->nw = 1 + (o->nso - 1) / 64;
  o->thr = thr;
  if (o->nw > MAXW) {
    snprintf(err, errlen, "more than %d words per determinant", MAXW);
    fclose(f);
    free(o);
    return NULL;
  }
  const size_t n = (size_t)o->nso;
  o->h1 = calloc(n * n, sizeof(double));
  o->g = calloc(n * n * n * n, sizeof(double));
  o->gset = calloc(n * n * n * n, 1);
  o->oe_idx = calloc(n, sizeof(int));
  o->oe_val = calloc(n, sizeof(double));
  double v;
  int i, a, j, b;
  while (fscanf(f, "%lf %d %d %d %d", &v, &i, &a, &j, &b) == 5) {
    if (i && a && j && b) {
      if (o->uhf) {
        ins(o, i - 1, j - 1, a - 1, b - 1, v);
        ins(o, i - 1, b - 1, a - 1, j - 1, v);
        ins(o, a - 1, j - 1, i - 1, b - 1, v);
        ins(o, a - 1, b - 1, i - 1, j - 1, v);
      } else {
        rhf_ins(o, i, j, a, b, v);
        rhf_ins(o, i, b, a, j, v);
        rhf_ins(o, a, j, i, b, v);
        rhf_ins(o, a, b, i, j, v);
      }
    } else if (a) {
      if (o->uhf) {
        o->h1[(i - 1) * n + (a - 1)] = v;
        o->h1[(a - 1) * n + (i - 1)] = v;
      } else {
        o->h1[(2 * i - 2) * n + (2 * a - 2)] = v;
        o->h1[(2 * i - 1) * n + (2 * a - 1)] = v;
        o->h1[(2 * a - 2) * n + (2 * i - 2)] = v;
        o->h1[(2 * a - 1) * n + (2 * i - 1)] = v;
      }
    } else if (i) {
      if (o->uhf) {
        add_oe(o, i - 1, v);
      } else {
        add_oe(o, 2 * i - 2, v);
        add_oe(o, 2 * i - 1, v);
      }
    } else {
      o->ecore = v;
    }
  }
  fclose(f);
  build_doubles(o);
  build_singles(o);
  build_diagonal(o);
  return o;
}

void oracle_free(oracle* o) {
  if (!o) return;
  const int n = o->nso;
  for (int x = 0; x < n * n; ++x) free(o->dbl[x]);
  for (int x = 0; x < n; ++x) {
    for (int y = 0; y < o->nsgl[x]; ++y) free(o->sgl[x][y].t);
    free(o->sgl[x]);
  }
  free(o->dbl);
  free(o->ndbl);
  free(o->sgl);
  free(o->nsgl);
  free(o->h1);
  free(o->g);
  free(o->gset);
  free(o->oe_idx);
  free(o->oe_val);
  free(o->d1);
  free(o->d2);
  free(o);
}

void oracle_info(const oracle* o, int32_t* nso, int32_t* nelec, int32_t* ms2, int32_t* nw, double* ecore) {
  *nso = o->nso;
  *nelec = o->nelec;
  *ms2 = o->ms2;
  *nw = o->nw;
  *ecore = o->ecore;
}

void oracle_integrals(const oracle* o, double* h1, double* g2) {
  const size_t n = (size_t)o->nso;
  memcpy(h1, o->h1, n * n * sizeof(double));
  memcpy(g2, o->g, n * n * n * n * sizeof(double));
}

/* ---- determinant helpers (interleaved layout) ---- */

static int occ_bit(const uint64_t* d, int i) { return (int)((d[i / 64] >> (i % 64)) & 1u); }
static void set_bit(uint64_t* d, int i) { d[i / 64] |= (uint64_t)1 << (i % 64); }
static void clr_bit(uint64_t* d, int i) { d[i / 64] &= ~((uint64_t)1 << (i % 64)); }

static void below_mask(int i, int nw, uint64_t* m) {
  for (int t = 0; t < nw; ++t) {
    if (t < i / 64)
      m[t] = ~(uint64_t)0;
    else if (t == i / 64)
      m[t] = ((uint64_t)1 << (i % 64)) - 1;
    else
      m[t] = 0;
  }
}

/* Determinant::parity: parity of the set bits in [min(i,a), max(i,a)). */
static int parity(const uint64_t* d, int nw, int i, int a) {
  uint64_t mi[MAXW], ma[MAXW];
  below_mask(i, nw, mi);
  below_mask(a, nw, ma);
  int r = 0;
  for (int t = 0; t < nw; ++t) r ^= __builtin_parityll(d[t] & (mi[t] ^ ma[t]));
  return r;
}

static int occupied_list(const oracle* o, const uint64_t* d, int* occ) {
  int c = 0;
  for (int t = 0; t < o->nw; ++t) {
    uint64_t w = d[t];
    while (w) {
      occ[c++] = __builtin_ctzll(w) + 64 * t;
      w &= w - 1;
    }
  }
  return c;
}

double oracle_diagonal(const oracle* o, const uint64_t* det) {
  int occ[128];
  const int c = occupied_list(o, det, occ);
  double v = 0.0;
  for (int x = 0; x < c; ++x) {
    v += o->d1[occ[x]];
    for (int y = x + 1; y < c; ++y) v += o->d2[occ[x] * o->nso + occ[y]];
  }
  return v + o->ecore;
}

static void push(const oracle* o, const uint64_t* d, double v, uint64_t* out, double* vals, int64_t* cnt,
                 int64_t cap) {
  if (*cnt < cap) {
    for (int t = 0; t < o->nw; ++t) out[*cnt * o->nw + t] = d[t];
    vals[*cnt] = v;
  }
  ++*cnt;
}

int64_t oracle_column(const oracle* o, const uint64_t* det, uint64_t* out, double* vals, int64_t cap) {
  const int nw = o->nw, n = o->nso;
  int occ[128];
  const int c = occupied_list(o, det, occ);
  int64_t cnt = 0;
  push(o, det, oracle_diagonal(o, det), out, vals, &cnt, cap);
  for (int x = 0; x < c; ++x) {
    const int i = occ[x];
    for (int e = 0; e < o->nsgl[i]; ++e) {
      const sentry* s = &o->sgl[i][e];
      if (occ_bit(det, s->a)) continue;
      double v = s->h;
      for (int y = 0; y < c; ++y) v += s->t[occ[y]];
      uint64_t nd[MAXW] = {0, 0};
      for (int t = 0; t < nw; ++t) nd[t] = det[t];
      clr_bit(nd, i);
      if (parity(nd, nw, i, s->a)) v = -v;
      set_bit(nd, s->a);
      push(o, nd, v, out, vals, &cnt, cap);
    }
  }
  for (int x = 0; x < c; ++x)
    for (int y = x + 1; y < c; ++y) {
      const int i = occ[x], j = occ[y];
      const dentry* L = o->dbl[i * n + j];
      for (int e = 0; e < o->ndbl[i * n + j]; ++e) {
        const int a = L[e].a, b = L[e].b;
        if (occ_bit(det, a) || occ_bit(det, b)) continue;
        double v = L[e].v;
        uint64_t nd[MAXW] = {0, 0};
        for (int t = 0; t < nw; ++t) nd[t] = det[t];
        clr_bit(nd, i);
        const int s1 = parity(nd, nw, i, a);
        set_bit(nd, a);
        clr_bit(nd, j);
        const int s2 = parity(nd, nw, j, b);
        set_bit(nd, b);
        if (s1 ^ s2) v = -v;
        push(o, nd, v, out, vals, &cnt, cap);
      }
    }
  return cnt;
}

double oracle_off_diagonal(const oracle* o, const uint64_t* d1, const uint64_t* d2) {
  const int nw = o->nw, n = o->nso;
  uint64_t x[MAXW], in1[MAXW], in2[MAXW];
  int pc = 0;
  for (int t = 0; t < nw; ++t) {
    x[t] = d1[t] ^ d2[t];
    in1[t] = x[t] & d1[t];
    in2[t] = x[t] & d2[t];
    pc += __builtin_popcountll(x[t]);
  }
  int ij[4], ab[4];
  const int ni = occupied_list(o, in1, ij), na = occupied_list(o, in2, ab);
  if (pc == 2 && ni == 1 && na == 1) {
    const int i = ij[0], a = ab[0];
    for (int e = 0; e < o->nsgl[i]; ++e) {
      const sentry* s = &o->sgl[i][e];
      if (s->a != a) continue;
      int occ[128];
      const int c = occupied_list(o, d1, occ);
      double v = s->h;
      for (int y = 0; y < c; ++y) v += s->t[occ[y]];
      uint64_t nd[MAXW] = {0, 0};
      for (int t = 0; t < nw; ++t) nd[t] = d1[t];
      clr_bit(nd, i);
      if (parity(nd, nw, i, a)) v = -v;
      return v;
    }
    return 0.0;
  }
  if (pc == 4 && ni == 2 && na == 2) {
    const int i = ij[0], j = ij[1];
    const dentry* L = o->dbl[i * n + j];
    for (int e = 0; e < o->ndbl[i * n + j]; ++e) {
      const int a = L[e].a, b = L[e].b;
      if ((a == ab[1] && b == ab[0]) || (a == ab[0] && b == ab[1])) {
        double v = L[e].v;
        uint64_t nd[MAXW] = {0, 0};
        for (int t = 0; t < nw; ++t) nd[t] = d1[t];
        clr_bit(nd, i);
        const int s1 = parity(nd, nw, i, a);
        set_bit(nd, a);
        clr_bit(nd, j);
        const int s2 = parity(nd, nw, j, b);
        if (s1 ^ s2) v = -v;
        return v;
      }
    }
  }
  return 0.0;
}

void oracle_hsub(const oracle* o, const uint64_t* dets, int32_t k, double* h) {
  const int nw = o->nw;
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) h[i * k + j] = oracle_off_diagonal(o, dets + i * nw, dets + j * nw);
  for (int i = 0; i < k; ++i) h[i * k + i] = oracle_diagonal(o, dets + i * nw);
}

void oracle_hartree_fock(const oracle* o, uint64_t* det) {
  const int n = o->nso;
  int m = o->n_oe;
  int* idx = malloc((size_t)(m > 0 ? m : n) * sizeof(int));
  double* en = malloc((size_t)(m > 0 ? m : n) * sizeof(double));
  if (m == 0) {
    m = n;
    for (int i = 0; i < n; ++i) {
      idx[i] = i;
      en[i] = i;
    }
  } else {
    memcpy(idx, o->oe_idx, m * sizeof(int));
    memcpy(en, o->oe_val, m * sizeof(double));
  }
  /* sort by energy, ties by spin-orbital index (insertion sort: m <= 128) */
  for (int x = 1; x < m; ++x) {
    const int ti = idx[x];
    const double te = en[x];
    int y = x - 1;
    while (y >= 0 && (en[y] > te || (en[y] == te && idx[y] > ti))) {
      idx[y + 1] = idx[y];
      en[y + 1] = en[y];
      --y;
    }
    idx[y + 1] = ti;
    en[y + 1] = te;
  }
  for (int t = 0; t < o->nw; ++t) det[t] = 0;
  const int n_alpha = (o->nelec + o->ms2) / 2, n_beta = (o->nelec - o->ms2) / 2;
  for (int i = 0, ia = 0, ib = 0; i < o->nelec && i < m; ++i) {
    const int orb = idx[i];
    if (orb % 2 == 0 && ia < n_alpha) {
      set_bit(det, orb);
      ++ia;
    } else if (orb % 2 == 1 && ib < n_beta) {
      set_bit(det, orb);
      ++ib;
    }
  }
  free(idx);
  free(en);
}
