/* Test infrastructure (oracle only) -- never linked into the product.
 * CPU restatement of the reference's kernel library, direct sum, octree and
 * interaction lists; see kifmm_oracle.h for the function-to-reference map.
 * Each function below names the reference lines it follows. */
#define _GNU_SOURCE
#include "kifmm_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ------------------------------------------------------------------------ */
/* Kernel library                                                            */
/* ------------------------------------------------------------------------ */

/* fmm3d/kernel3d.cpp:24-86 */
int ko_kernel_dofs(int kt, int* sdof, int* tdof) {
  int s = 0, t = 0;
  switch (kt) {
    case 111: case 121: s = 1; t = 1; break;
    case 301: s = 4; t = 3; break;
    case 311: case 321: s = 3; t = 3; break;
    case 312: case 322: s = 3; t = 1; break;
    case 511: case 521: s = 3; t = 3; break;
    default: return -1;
  }
  *sdof = s;
  *tdof = t;
  return 0;
}

/* Interaction block of one (target, source) pair, row-major [tdof][sdof],
 * following the per-kernel formulas of fmm3d/kernel3d.cpp:116-369 including
 * the singular cut-off r < 1e-8 -> 0 (fmm3d/kernel3d.cpp:21). */
static void kernel_block(int kt, const double* coefs, const double* tp, const double* sp,
                         const double* sn, double* blk) {
  const double mindif = 1e-8;
  double x = tp[0] - sp[0], y = tp[1] - sp[1], z = tp[2] - sp[2];
  double r2 = x * x + y * y + z * z;
  double r = sqrt(r2);
  int sd = 0, td = 0;
  ko_kernel_dofs(kt, &sd, &td);
  if (r < mindif) {
    for (int i = 0; i < sd * td; i++) blk[i] = 0.0;
    return;
  }
  double d[3] = {x, y, z};
  if (kt == 111) { /* :124-138 */
    blk[0] = (1.0 / (4.0 * M_PI)) / r;
  } else if (kt == 121) { /* :139-154 */
    double rn = x * sn[0] + y * sn[1] + z * sn[2];
    double r3 = r2 * r;
    blk[0] = -(1.0 / (4.0 * M_PI)) / r3 * rn;
  } else if (kt == 301) { /* :160-184 */
    double mu = coefs[0];
    double r3 = r2 * r;
    double G = (1.0 / mu) * (1.0 / (8.0 * M_PI)) / r;
    double H = (1.0 / mu) * (1.0 / (8.0 * M_PI)) / r3;
    double A = (1.0 / (4.0 * M_PI)) / r3;
    for (int a = 0; a < 3; a++) {
      for (int b = 0; b < 3; b++) blk[a * 4 + b] = (a == b ? G : 0.0) + H * d[a] * d[b];
      blk[a * 4 + 3] = A * d[a];
    }
  } else if (kt == 311) { /* :185-205 */
    double oomu = 1.0 / coefs[0];
    double r3 = r2 * r;
    double G = (1.0 / (8.0 * M_PI)) / r;
    double H = (1.0 / (8.0 * M_PI)) / r3;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) blk[a * 3 + b] = oomu * ((a == b ? G : 0.0) + H * d[a] * d[b]);
  } else if (kt == 312) { /* :206-221 */
    double r3 = r2 * r;
    for (int b = 0; b < 3; b++) blk[b] = (1.0 / (4.0 * M_PI)) * d[b] / r3;
  } else if (kt == 321) { /* :222-242 */
    double rn = x * sn[0] + y * sn[1] + z * sn[2];
    double r5 = r2 * r2 * r;
    double C = -(6.0 / (8.0 * M_PI)) / r5;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) blk[a * 3 + b] = C * rn * d[a] * d[b];
  } else if (kt == 322) { /* :243-265 */
    double mu = coefs[0];
    double coef = mu * (1.0 / (2.0 * M_PI));
    double rn = x * sn[0] + y * sn[1] + z * sn[2];
    double r3 = r2 * r;
    double r5 = r3 * r2;
    for (int b = 0; b < 3; b++) blk[b] = coef * (sn[b] / r3 - 3 * rn * d[b] / r5);
  } else if (kt == 511) { /* :315-337 */
    double mu = coefs[0], ve = coefs[1];
    double sc1 = (3.0 - 4.0 * ve) / (16.0 * M_PI * (1.0 - ve));
    double sc2 = 1.0 / (16.0 * M_PI * (1.0 - ve));
    double oomu = 1.0 / mu;
    double r3 = r2 * r;
    double G = sc1 / r;
    double H = sc2 / r3;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) blk[a * 3 + b] = oomu * ((a == b ? G : 0.0) + H * d[a] * d[b]);
  } else if (kt == 521) { /* :338-369 */
    double ve = coefs[1];
    double dc1 = -(1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve));
    double dc2 = (1 - 2.0 * ve) / (8.0 * M_PI * (1.0 - ve));
    double dc3 = -3.0 / (8.0 * M_PI * (1.0 - ve));
    double rn = x * sn[0] + y * sn[1] + z * sn[2];
    double r3 = r2 * r;
    double r5 = r3 * r2;
    double A = dc1 / r3, B = dc2 / r3, C = dc3 / r5;
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++)
        blk[a * 3 + b] = A * ((a == b ? rn : 0.0) + sn[a] * d[b]) + B * (d[a] * sn[b]) + C * rn * d[a] * d[b];
  }
}

typedef struct {
  int kt;
  const double* coefs;
  int ns, nt, sd, td;
  const double *sp, *sn, *den, *tp;
  double* out;
  int t0, t1;
} direct_job;

static void* direct_worker(void* arg) {
  direct_job* j = (direct_job*)arg;
  double blk[16];
  for (int t = j->t0; t < j->t1; t++) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < j->ns; s++) {
      kernel_block(j->kt, j->coefs, j->tp + 3 * (size_t)t, j->sp + 3 * (size_t)s, j->sn + 3 * (size_t)s, blk);
      const double* f = j->den + (size_t)s * j->sd;
      for (int a = 0; a < j->td; a++)
        for (int b = 0; b < j->sd; b++) acc[a] += blk[a * j->sd + b] * f[b];
    }
    for (int a = 0; a < j->td; a++) j->out[(size_t)t * j->td + a] = acc[a];
  }
  return NULL;
}

/* Dense3d::eval, fmm3d/dense3d.cpp:38-57 (one target row block at a time,
 * then y = inter * den). */
int ko_direct(int kt, int ncoef, const double* coefs, int ns, const double* srcpos,
              const double* srcnor, const double* srcden, int nt, const double* trgpos,
              double* trgval, int nthreads) {
  int sd, td;
  if (ko_kernel_dofs(kt, &sd, &td) != 0) return -1;
  if ((kt == 301 || kt == 311 || kt == 321 || kt == 322) && ncoef < 1) return -1;
  if ((kt == 511 || kt == 521) && ncoef < 2) return -1;
  if (nthreads <= 0) nthreads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (nthreads < 1) nthreads = 1;
  if (nthreads > nt) nthreads = nt > 0 ? nt : 1;
  direct_job* jobs = (direct_job*)calloc((size_t)nthreads, sizeof(direct_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int i = 0; i < nthreads; i++) {
    direct_job* j = &jobs[i];
    j->kt = kt; j->coefs = coefs; j->ns = ns; j->nt = nt; j->sd = sd; j->td = td;
    j->sp = srcpos; j->sn = srcnor; j->den = srcden; j->tp = trgpos; j->out = trgval;
    j->t0 = (int)((long)nt * i / nthreads);
    j->t1 = (int)((long)nt * (i + 1) / nthreads);
    pthread_create(&th[i], NULL, direct_worker, j);
  }
  for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
  free(jobs);
  free(th);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Octree and interaction lists                                             */
/* ------------------------------------------------------------------------ */

typedef struct {
  int* a;
  int n, cap;
} ivec;

static void iv_push(ivec* v, int x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? 2 * v->cap : 8;
    v->a = (int*)realloc(v->a, sizeof(int) * (size_t)v->cap);
  }
  v->a[v->n++] = x;
}

static void iv_free(ivec* v) {
  free(v->a);
  v->a = NULL;
  v->n = v->cap = 0;
}

static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

enum { KO_SRC = 1, KO_TRG = 2 };

struct ko_tree {
  int n, cap;
  int *par, *chd, *path, *depth, *tag, *sbeg, *snum, *tbeg, *tnum;
  int *scnt, *tcnt; /* lsmvec of srcdata/trgdata: counts kept after a split */
  ivec* svis;
  ivec* tvis;
  ivec* lists[4];
  double ctr[3];
  int rootlvl, ptsmax, maxlevel;
};

static int add_node(ko_tree* t, int par, int p0, int p1, int p2, int depth) {
  if (t->n == t->cap) {
    t->cap = t->cap ? 2 * t->cap : 64;
    size_t c = (size_t)t->cap;
    t->par = (int*)realloc(t->par, sizeof(int) * c);
    t->chd = (int*)realloc(t->chd, sizeof(int) * c);
    t->path = (int*)realloc(t->path, sizeof(int) * 3 * c);
    t->depth = (int*)realloc(t->depth, sizeof(int) * c);
    t->tag = (int*)realloc(t->tag, sizeof(int) * c);
    t->sbeg = (int*)realloc(t->sbeg, sizeof(int) * c);
    t->snum = (int*)realloc(t->snum, sizeof(int) * c);
    t->tbeg = (int*)realloc(t->tbeg, sizeof(int) * c);
    t->tnum = (int*)realloc(t->tnum, sizeof(int) * c);
    t->scnt = (int*)realloc(t->scnt, sizeof(int) * c);
    t->tcnt = (int*)realloc(t->tcnt, sizeof(int) * c);
    t->svis = (ivec*)realloc(t->svis, sizeof(ivec) * c);
    t->tvis = (ivec*)realloc(t->tvis, sizeof(ivec) * c);
    for (int l = 0; l < 4; l++) t->lists[l] = (ivec*)realloc(t->lists[l], sizeof(ivec) * c);
  }
  int g = t->n++;
  t->par[g] = par;
  t->chd[g] = -1;
  t->path[3 * g] = p0;
  t->path[3 * g + 1] = p1;
  t->path[3 * g + 2] = p2;
  t->depth[g] = depth;
  t->tag[g] = 0;
  t->sbeg[g] = t->snum[g] = t->tbeg[g] = t->tnum[g] = 0;
  t->scnt[g] = t->tcnt[g] = 0;
  memset(&t->svis[g], 0, sizeof(ivec));
  memset(&t->tvis[g], 0, sizeof(ivec));
  for (int l = 0; l < 4; l++) memset(&t->lists[l][g], 0, sizeof(ivec));
  return g;
}

static double root_rad(const ko_tree* t) { return pow(2.0, -t->rootlvl); } /* let3d.hpp:98 */

/* Let3d::center, fmm3d/let3d.cpp:309-318 */
static void node_center(const ko_tree* t, int g, double c[3]) {
  double rad = root_rad(t);
  int tmp = 1 << t->depth[g];
  for (int d = 0; d < 3; d++) {
    double ll = t->ctr[d] - rad;
    c[d] = ll + (2 * rad) * (t->path[3 * g + d] + 0.5) / (double)tmp;
  }
}

/* child index order a*4 + b*2 + c, fmm3d/let3d.cpp:304-308 */
static int child_of(const ko_tree* t, int g, int a, int b, int c) { return t->chd[g] + a * 4 + b * 2 + c; }

static int in_box(const ko_tree* t, const double* p) {
  double rad = root_rad(t);
  for (int d = 0; d < 3; d++) {
    double lo = t->ctr[d] - rad, hi = t->ctr[d] + rad;
    if (!(p[d] >= lo && p[d] <= hi)) return 0;
  }
  return 1;
}

/* distribute the point ids of node g among its children (let3d.cpp:96-106) */
static void split_points(ko_tree* t, int g, ivec* vis, const double* pos) {
  double c[3];
  node_center(t, g, c);
  ivec* v = &vis[g];
  for (int k = 0; k < v->n; k++) {
    const double* p = pos + 3 * (size_t)v->a[k];
    int a = p[0] >= c[0], b = p[1] >= c[1], cc = p[2] >= c[2];
    iv_push(&vis[child_of(t, g, a, b, cc)], v->a[k]);
  }
  iv_free(v);
  int* cnt = (vis == t->svis) ? t->scnt : t->tcnt;
  for (int o = 0; o < 8; o++) cnt[t->chd[g] + o] = vis[t->chd[g] + o].n;
}

/* Let3d::findgnt, fmm3d/let3d.cpp:325-337 */
static int findgnt(const ko_tree* t, int wdepth, const int wpath[3]) {
  int cur = 0;
  int left[3] = {wpath[0], wpath[1], wpath[2]};
  while (t->depth[cur] < wdepth && t->chd[cur] != -1) {
    int dif = wdepth - t->depth[cur];
    int tmp = 1 << (dif - 1);
    int ch[3];
    for (int d = 0; d < 3; d++) {
      ch[d] = left[d] / tmp;
      left[d] -= ch[d] * tmp;
    }
    cur = child_of(t, cur, ch[0], ch[1], ch[2]);
  }
  return cur;
}

/* Let3d::adjacent, fmm3d/let3d.cpp:339-352 */
static int adjacent(const ko_tree* t, int me, int yo) {
  int md = t->depth[me] > t->depth[yo] ? t->depth[me] : t->depth[yo];
  int merad = 1 << (md - t->depth[me]);
  int yorad = 1 << (md - t->depth[yo]);
  int rad = merad + yorad;
  int all_le = 1, mx = 0;
  for (int d = 0; d < 3; d++) {
    int mc = (2 * t->path[3 * me + d] + 1) * merad;
    int yc = (2 * t->path[3 * yo + d] + 1) * yorad;
    int dif = abs(mc - yc);
    if (dif > rad) all_le = 0;
    if (dif > mx) mx = dif;
  }
  return all_le && mx == rad;
}

static void finish_list(ko_tree* t, ivec* set, ivec* out) {
  /* std::set semantics: sorted, unique; keep source nodes only (let3d.cpp:272-279) */
  if (set->n > 1) qsort(set->a, (size_t)set->n, sizeof(int), cmp_int);
  int last = -1;
  for (int k = 0; k < set->n; k++) {
    int g = set->a[k];
    if (g == last) continue;
    last = g;
    if (t->tag[g] & KO_SRC) iv_push(out, g);
  }
  iv_free(set);
}

/* Let3d::calgnext, fmm3d/let3d.cpp:214-281 */
static void calgnext(ko_tree* t, int g) {
  ivec U = {0}, V = {0}, W = {0}, X = {0};
  int term = t->chd[g] == -1;
  if (t->par[g] != -1) {
    int pg = t->par[g];
    int maxidx = 1 << t->depth[g];
    ivec queue = {0};
    for (int i = -2; i < 4; i++)
      for (int j = -2; j < 4; j++)
        for (int k = -2; k < 4; k++) {
          int tp[3] = {2 * t->path[3 * pg] + i, 2 * t->path[3 * pg + 1] + j, 2 * t->path[3 * pg + 2] + k};
          int ok = 1;
          for (int d = 0; d < 3; d++)
            if (!(tp[d] >= 0 && tp[d] < maxidx)) ok = 0;
          if (!ok) continue;
          if (tp[0] == t->path[3 * g] && tp[1] == t->path[3 * g + 1] && tp[2] == t->path[3 * g + 2]) continue;
          int res = findgnt(t, t->depth[g], tp);
          int adj = adjacent(t, res, g);
          if (t->depth[res] < t->depth[g]) {
            if (adj) {
              if (term) iv_push(&U, res);
            } else {
              iv_push(&X, res);
            }
          }
          if (t->depth[res] == t->depth[g]) {
            if (!adj) {
              iv_push(&V, res);
            } else if (term) {
              queue.n = 0;
              iv_push(&queue, res);
              for (int qh = 0; qh < queue.n; qh++) {
                int f = queue.a[qh];
                if (!adjacent(t, f, g)) {
                  iv_push(&W, f);
                } else if (t->chd[f] == -1) {
                  iv_push(&U, f);
                } else {
                  for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++)
                      for (int c = 0; c < 2; c++) iv_push(&queue, child_of(t, f, a, b, c));
                }
              }
            }
          }
        }
    iv_free(&queue);
  }
  if (term) iv_push(&U, g);
  finish_list(t, &U, &t->lists[0][g]);
  finish_list(t, &V, &t->lists[1][g]);
  finish_list(t, &W, &t->lists[2][g]);
  finish_list(t, &X, &t->lists[3][g]);
}

ko_tree* ko_tree_build(int ptsmax, int maxlevel, const double* ctr, int rootlvl, int ns,
                       const double* srcpos, int nt, const double* trgpos, int* status) {
  ko_tree* t = (ko_tree*)calloc(1, sizeof(ko_tree));
  t->ctr[0] = ctr[0];
  t->ctr[1] = ctr[1];
  t->ctr[2] = ctr[2];
  t->rootlvl = rootlvl;
  t->ptsmax = ptsmax;
  t->maxlevel = maxlevel;
  *status = 0;
  /* Let3d::srcdata, fmm3d/let3d.cpp:56-137 */
  add_node(t, -1, 0, 0, 0, 0);
  for (int k = 0; k < ns; k++) {
    if (!in_box(t, srcpos + 3 * (size_t)k)) *status = 3;
    iv_push(&t->svis[0], k);
  }
  if (*status) return t;
  t->scnt[0] = ns;
  int level = 0, arrbeg = 0, arrend = 1;
  while (arrbeg < arrend) {
    int arrcnt = arrend;
    for (int k = arrbeg; k < arrend; k++) {
      if (t->scnt[k] > ptsmax && level < maxlevel - 1) {
        t->chd[k] = arrcnt;
        arrcnt += 8;
        for (int a = 0; a < 2; a++)
          for (int b = 0; b < 2; b++)
            for (int c = 0; c < 2; c++)
              add_node(t, k, 2 * t->path[3 * k] + a, 2 * t->path[3 * k + 1] + b, 2 * t->path[3 * k + 2] + c,
                       t->depth[k] + 1);
        split_points(t, k, t->svis, srcpos);
      }
    }
    level++;
    arrbeg = arrend;
    arrend = arrcnt;
  }
  int sum = 0;
  for (int g = 0; g < t->n; g++) {
    if (t->scnt[g] > 0) {
      t->tag[g] |= KO_SRC;
      if (t->chd[g] == -1) {
        t->sbeg[g] = sum;
        t->snum[g] = t->scnt[g];
        sum += t->scnt[g];
      }
    }
  }
  /* Let3d::trgdata, fmm3d/let3d.cpp:140-211 */
  for (int k = 0; k < nt; k++) {
    if (!in_box(t, trgpos + 3 * (size_t)k)) *status = 3;
    iv_push(&t->tvis[0], k);
  }
  if (*status) return t;
  t->tcnt[0] = nt;
  for (int g = 0; g < t->n; g++)
    if (t->chd[g] != -1) split_points(t, g, t->tvis, trgpos);
  sum = 0;
  for (int g = 0; g < t->n; g++) {
    if (t->tcnt[g] > 0) {
      t->tag[g] |= KO_TRG;
      if (t->chd[g] == -1) {
        t->tbeg[g] = sum;
        t->tnum[g] = t->tcnt[g];
        sum += t->tcnt[g];
      }
    }
  }
  for (int g = 0; g < t->n; g++)
    if (t->tag[g] & KO_TRG) calgnext(t, g);
  return t;
}

int ko_tree_nnodes(const ko_tree* t) { return t->n; }

int ko_tree_nodes(const ko_tree* t, int* depth, int* path, int* par, int* chd, int* tag, int* sbeg,
                  int* snum, int* tbeg, int* tnum) {
  for (int g = 0; g < t->n; g++) {
    depth[g] = t->depth[g];
    path[3 * g] = t->path[3 * g];
    path[3 * g + 1] = t->path[3 * g + 1];
    path[3 * g + 2] = t->path[3 * g + 2];
    par[g] = t->par[g];
    chd[g] = t->chd[g];
    tag[g] = t->tag[g];
    sbeg[g] = t->sbeg[g];
    snum[g] = t->snum[g];
    tbeg[g] = t->tbeg[g];
    tnum[g] = t->tnum[g];
  }
  return 0;
}

static const ivec* pick(const ko_tree* t, int which, int g) {
  if (which < 4) return &t->lists[which][g];
  return which == 4 ? &t->svis[g] : &t->tvis[g];
}

long ko_tree_list_total(const ko_tree* t, int which) {
  long tot = 0;
  for (int g = 0; g < t->n; g++) tot += pick(t, which, g)->n;
  return tot;
}

int ko_tree_lists(const ko_tree* t, int which, long* ptr, int* idx) {
  long pos = 0;
  for (int g = 0; g < t->n; g++) {
    ptr[g] = pos;
    const ivec* v = pick(t, which, g);
    for (int k = 0; k < v->n; k++) idx[pos++] = v->a[k];
  }
  ptr[t->n] = pos;
  return 0;
}

void ko_tree_free(ko_tree* t) {
  if (!t) return;
  for (int g = 0; g < t->n; g++) {
    iv_free(&t->svis[g]);
    iv_free(&t->tvis[g]);
    for (int l = 0; l < 4; l++) iv_free(&t->lists[l][g]);
  }
  free(t->par); free(t->chd); free(t->path); free(t->depth); free(t->tag);
  free(t->sbeg); free(t->snum); free(t->tbeg); free(t->tnum);
  free(t->scnt); free(t->tcnt);
  free(t->svis); free(t->tvis);
  for (int l = 0; l < 4; l++) free(t->lists[l]);
  free(t);
}
