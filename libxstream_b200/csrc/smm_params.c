/*
 * Kernel-parameter table for the FP64 stack kernel: tuned records keyed by (type, m, n, k), read
 * from and written to a semicolon-separated CSV whose leading columns are the reference's
 * (DEVICE;TYPEID;M;N;K;S;GFLOPS, samples/smm/params/tune_multiply_*.csv line 1 and
 * samples/smm/smm_params.c:89-270), followed by this library's tunables (L;MT;NT;KP;WPB).
 * Replaces the reference's registry of JIT-ed kernels (samples/smm/smm_kernel.c:109-150): nothing
 * is compiled at run time, a record only selects one of the precompiled kernel variants.
 */
#include "internal.h"
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define XS_PARAMS_CAP 8192 /* power of two */

typedef struct xs_record_t {
  int used, type, m, n, k;
  double gflops;
  xs_smm_params_t p;
} xs_record_t;

static xs_record_t xs_table[XS_PARAMS_CAP];
static pthread_rwlock_t xs_table_lock = PTHREAD_RWLOCK_INITIALIZER;

static unsigned xs_hash(int type, int m, int n, int k) {
  unsigned h = 2166136261u;
  h = (h ^ (unsigned)type) * 16777619u;
  h = (h ^ (unsigned)m) * 16777619u;
  h = (h ^ (unsigned)n) * 16777619u;
  h = (h ^ (unsigned)k) * 16777619u;
  return h;
}

static int xs_clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static void xs_sanitize(xs_smm_params_t* p) {
  p->chunk = xs_clamp(p->chunk, 0, 1 << 20); /* 0: sized per stack by the launcher */
  p->mt = xs_clamp(p->mt, 1, 4);
  p->nt = xs_clamp(p->nt, 1, 4);
  p->kp = xs_clamp(p->kp, XS_KP_FMA, 4); /* 0: staged kernel (where compiled for the shape); -1: FMA kernel */
  p->generic = (0 != p->generic) ? 1 : 0;
  p->wpb = xs_clamp(p->wpb, 1, 16); /* above 4: consumer warps of a warp-specialised kernel */
  p->sorted = (0 != p->sorted) ? 1 : 0;
}

/* Tiles of at most 4x4 DMMA fragments per warp; prefer the split of ceil(x/8) fragments into
   equal sub-tiles with the least padding. */
static int xs_pick_tiles(int dim) {
  const int frags = (dim + 7) / 8;
  int best = 1, bestwaste = 1 << 30, t;
  for (t = 4; t >= 1; --t) {
    const int nsub = (frags + t - 1) / t;
    const int waste = nsub * t - frags;
    if (waste < bestwaste) {
      bestwaste = waste;
      best = t;
    }
  }
  return best;
}

void xs_params_default(int m, int n, int k, int stack_size, xs_smm_params_t* out) {
  const int mt = xs_pick_tiles(m), nt = xs_pick_tiles(n);
  (void)stack_size;
  out->chunk = 0; /* open: the launcher sizes chunks to one wave of resident CTAs */
  out->mt = mt;
  out->nt = nt;
  out->kp = ((k + 3) / 4 <= 2) ? 2 : 4;
  out->wpb = 4;
  out->sorted = 0;
  out->generic = 0;
  { /* prefer a shape-specialised kernel with the same tiles (the first one listed) */
    int triples[3 * 8], i;
    const int nspec = xs_smm_f64_specialized(m, n, k, triples, 8);
    for (i = 0; i < nspec && i < 8; ++i) {
      if (triples[3 * i] == mt && triples[3 * i + 1] == nt) {
        out->kp = triples[3 * i + 2];
        break;
      }
    }
  }
  xs_sanitize(out);
}

static float xs_mlp_minconf(void) {
  static float v = -1.f;
  if (0 > v) {
    const char* const env = getenv("LIBXSTREAM_B200_MLP_MINCONF");
    v = (NULL != env) ? (float)atof(env) : 0.5f;
    if (0 > v) v = 0.f;
  }
  return v;
}

void xs_params_lookup(int type, int m, int n, int k, int stack_size, xs_smm_params_t* out) {
  xs_params_lookup_ex(type, m, n, k, stack_size, out, NULL);
}

void xs_params_lookup_ex(int type, int m, int n, int k, int stack_size, xs_smm_params_t* out, int* source) {
  unsigned h = xs_hash(type, m, n, k) & (XS_PARAMS_CAP - 1);
  int probe, found = 0;
  pthread_rwlock_rdlock(&xs_table_lock);
  for (probe = 0; probe < XS_PARAMS_CAP; ++probe) {
    const xs_record_t* const r = &xs_table[(h + probe) & (XS_PARAMS_CAP - 1)];
    if (!r->used) break;
    if (r->type == type && r->m == m && r->n == n && r->k == k) {
      *out = r->p;
      found = 1;
      break;
    }
  }
  pthread_rwlock_unlock(&xs_table_lock);
  if (NULL != source) *source = found ? XS_PARAMS_TUNED : XS_PARAMS_DEFAULT;
  if (!found) {
    int mt, nt, kp;
    float conf = 0.f;
    xs_params_default(m, n, k, stack_size, out);
    if (xs_mlp_lookup(m, n, k, stack_size, &mt, &nt, &kp, &conf)) {
      /* the prediction beats the default heuristic even when unconfident; the confidence only decides
         whether the exhaustive tuner should check it (LIBXSTREAM_B200_AUTOTUNE) */
      out->mt = mt;
      out->nt = nt;
      out->kp = kp;
      out->chunk = 0;
      out->wpb = 4;
      out->generic = 0;
      xs_sanitize(out);
      if (NULL != source) *source = (conf >= xs_mlp_minconf()) ? XS_PARAMS_PREDICTED : XS_PARAMS_LOWCONF;
    }
    if (XS_KP_FMA != out->kp) { /* a staged kernel compiled for the shape (listed with kp = 0) beat the
         register kernel's configurations where it was measured: its whole-block tile replaces heuristic
         and predicted DMMA tiles (tuned records and a predicted FMA kernel stay; the tuner times the
         staged kernel under its whole-block tile, so the predictor learned it against the FMA kernel) */
      int triples[3 * 8], i;
      const int nspec = xs_smm_f64_specialized(m, n, k, triples, 8);
      for (i = 0; i < nspec && i < 8; ++i) {
        if (0 == triples[3 * i + 2]) {
          out->mt = triples[3 * i];
          out->nt = triples[3 * i + 1];
          out->kp = 0;
          break;
        }
      }
    }
  }
}

int xs_params_set(int type, int m, int n, int k, const xs_smm_params_t* p, double gflops) {
  unsigned h = xs_hash(type, m, n, k) & (XS_PARAMS_CAP - 1);
  int probe, result = -1;
  pthread_rwlock_wrlock(&xs_table_lock);
  for (probe = 0; probe < XS_PARAMS_CAP; ++probe) {
    xs_record_t* const r = &xs_table[(h + probe) & (XS_PARAMS_CAP - 1)];
    if (!r->used || (r->type == type && r->m == m && r->n == n && r->k == k)) {
      if (!r->used || gflops >= r->gflops || 0 >= gflops) {
        r->used = 1;
        r->type = type;
        r->m = m;
        r->n = n;
        r->k = k;
        r->gflops = gflops;
        r->p = *p;
        xs_sanitize(&r->p);
      }
      result = 0;
      break;
    }
  }
  pthread_rwlock_unlock(&xs_table_lock);
  return result;
}

void xs_params_clear(void) {
  pthread_rwlock_wrlock(&xs_table_lock);
  memset(xs_table, 0, sizeof(xs_table));
  pthread_rwlock_unlock(&xs_table_lock);
}

/* CSV: DEVICE;TYPEID;M;N;K;S;GFLOPS;L;MT;NT;KP;WPB[;GEN] (the first line is a header). */
int xs_params_load_csv(const char* path) {
  char line[1024];
  int count = 0, lineno = 0;
  FILE* const f = (NULL != path) ? fopen(path, "r") : NULL;
  if (NULL == f) return -1;
  while (NULL != fgets(line, sizeof(line), f)) {
    char* fields[16];
    int nf = 0;
    char* tok = strtok(line, ";\n\r");
    ++lineno;
    while (NULL != tok && nf < 16) {
      fields[nf++] = tok;
      tok = strtok(NULL, ";\n\r");
    }
    if (1 == lineno && 0 < nf && NULL != strstr(fields[0], "DEVICE")) continue; /* header */
    if (12 <= nf) {
      xs_smm_params_t p;
      const int type = atoi(fields[1]), m = atoi(fields[2]), n = atoi(fields[3]), k = atoi(fields[4]);
      const double gflops = atof(fields[6]);
      p.chunk = atoi(fields[7]);
      p.mt = atoi(fields[8]);
      p.nt = atoi(fields[9]);
      p.kp = atoi(fields[10]);
      p.wpb = atoi(fields[11]);
      p.sorted = 0;
      p.generic = (13 <= nf) ? atoi(fields[12]) : 0;
      if (0 < m && 0 < n && 0 < k && 0 == xs_params_set(type, m, n, k, &p, gflops)) ++count;
    }
  }
  fclose(f);
  return count;
}
