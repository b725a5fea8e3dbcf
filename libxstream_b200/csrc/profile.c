/*
 * Per-kernel launch profile: when enabled (LIBXSTREAM_B200_PROFILE=1 or
 * libxstream_b200_profile_enable(1)), every launch site records a pair of timing events around its
 * kernel on the launch stream, together with the work the launch states (flops and bytes). The
 * pairs are resolved lazily on query, so profiling adds no host synchronisation to the launches.
 * Counterpart of the reference's per-kernel {ms, gflop, mb} histogram filled from OpenCL profiling
 * events (src/libxstream.c:2629-2723, enabled by LIBXSTREAM_PROFILE, src/libxstream_stream.c:110-114).
 */
#include "internal.h"
#include "../../include/libxstream_b200.h"
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define XS_PROF_KINDS 16
#define XS_PROF_PENDING 8192

typedef struct xs_prof_pair_t {
  cudaEvent_t start, stop;
  int kind;
  double flops, bytes;
} xs_prof_pair_t;

typedef struct xs_prof_total_t {
  char name[32];
  long launches;
  double ms, flops, bytes;
} xs_prof_total_t;

static pthread_mutex_t xs_prof_lock = PTHREAD_MUTEX_INITIALIZER;
static int xs_prof_on = -1;
static xs_prof_total_t xs_prof_totals[XS_PROF_KINDS];
static int xs_prof_nkinds = 0;
static xs_prof_pair_t xs_prof_pending[XS_PROF_PENDING];
static int xs_prof_npending = 0;

int xs_profile_enabled(void) {
  if (0 > xs_prof_on) {
    const char* const env = getenv("LIBXSTREAM_B200_PROFILE");
    xs_prof_on = (NULL != env && '\0' != *env && '0' != *env) ? 1 : 0;
  }
  return xs_prof_on;
}

static int xs_prof_kind(const char* name) {
  int i;
  for (i = 0; i < xs_prof_nkinds; ++i) {
    if (0 == strncmp(xs_prof_totals[i].name, name, sizeof(xs_prof_totals[i].name) - 1)) return i;
  }
  if (xs_prof_nkinds < XS_PROF_KINDS) {
    memset(&xs_prof_totals[xs_prof_nkinds], 0, sizeof(xs_prof_total_t));
    strncpy(xs_prof_totals[xs_prof_nkinds].name, name, sizeof(xs_prof_totals[0].name) - 1);
    return xs_prof_nkinds++;
  }
  return -1;
}

/* Resolve every pending pair (waits for their stop events); caller holds the lock. */
static void xs_prof_drain(void) {
  int i;
  for (i = 0; i < xs_prof_npending; ++i) {
    xs_prof_pair_t* const p = &xs_prof_pending[i];
    float ms = 0.f;
    if (cudaSuccess == cudaEventSynchronize(p->stop) && cudaSuccess == cudaEventElapsedTime(&ms, p->start, p->stop)) {
      xs_prof_total_t* const t = &xs_prof_totals[p->kind];
      t->launches += 1;
      t->ms += ms;
      t->flops += p->flops;
      t->bytes += p->bytes;
    }
    cudaEventDestroy(p->start);
    cudaEventDestroy(p->stop);
  }
  xs_prof_npending = 0;
}

void* xs_profile_begin(void* stream) {
  cudaEvent_t e = NULL;
  if (!xs_profile_enabled()) return NULL;
  if (cudaSuccess != cudaEventCreate(&e)) return NULL;
  if (cudaSuccess != cudaEventRecord(e, (cudaStream_t)stream)) {
    cudaEventDestroy(e);
    return NULL;
  }
  return (void*)e;
}

void xs_profile_end(void* token, const char* name, double flops, double bytes, void* stream) {
  cudaEvent_t stop = NULL;
  int kind;
  if (NULL == token) return;
  if (cudaSuccess != cudaEventCreate(&stop) || cudaSuccess != cudaEventRecord(stop, (cudaStream_t)stream)) {
    cudaEventDestroy((cudaEvent_t)token);
    if (NULL != stop) cudaEventDestroy(stop);
    return;
  }
  pthread_mutex_lock(&xs_prof_lock);
  kind = xs_prof_kind(name);
  if (XS_PROF_PENDING == xs_prof_npending) xs_prof_drain();
  if (0 <= kind) {
    xs_prof_pair_t* const p = &xs_prof_pending[xs_prof_npending++];
    p->start = (cudaEvent_t)token;
    p->stop = stop;
    p->kind = kind;
    p->flops = flops;
    p->bytes = bytes;
  }
  else {
    cudaEventDestroy((cudaEvent_t)token);
    cudaEventDestroy(stop);
  }
  pthread_mutex_unlock(&xs_prof_lock);
}

void libxstream_b200_profile_enable(int on) { xs_prof_on = (0 != on) ? 1 : 0; }

void libxstream_b200_profile_reset(void) {
  pthread_mutex_lock(&xs_prof_lock);
  xs_prof_drain();
  memset(xs_prof_totals, 0, sizeof(xs_prof_totals));
  xs_prof_nkinds = 0;
  pthread_mutex_unlock(&xs_prof_lock);
}

int libxstream_b200_profile_query(const char* kernel, long* launches, double* ms, double* gflop, double* gbyte) {
  int i, found = -1;
  pthread_mutex_lock(&xs_prof_lock);
  xs_prof_drain();
  for (i = 0; i < xs_prof_nkinds; ++i) {
    if (NULL != kernel && 0 == strcmp(xs_prof_totals[i].name, kernel)) found = i;
  }
  if (0 <= found) {
    if (NULL != launches) *launches = xs_prof_totals[found].launches;
    if (NULL != ms) *ms = xs_prof_totals[found].ms;
    if (NULL != gflop) *gflop = xs_prof_totals[found].flops * 1e-9;
    if (NULL != gbyte) *gbyte = xs_prof_totals[found].bytes * 1e-9;
  }
  pthread_mutex_unlock(&xs_prof_lock);
  return (0 <= found) ? 0 : -1;
}

int libxstream_b200_profile_kernels(char* names, int capacity) {
  int i, used = 0;
  if (NULL == names || 0 >= capacity) return -1;
  names[0] = '\0';
  pthread_mutex_lock(&xs_prof_lock);
  for (i = 0; i < xs_prof_nkinds; ++i) {
    const int len = (int)strlen(xs_prof_totals[i].name);
    if (used + len + 2 > capacity) break;
    memcpy(names + used, xs_prof_totals[i].name, (size_t)len);
    used += len;
    names[used++] = ';';
    names[used] = '\0';
  }
  pthread_mutex_unlock(&xs_prof_lock);
  return used;
}

int libxstream_b200_event_create_timed(void** event_p) {
  cudaEvent_t e = NULL;
  int r;
  if (NULL == event_p) return EXIT_FAILURE;
  *event_p = NULL;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  r = (int)cudaEventCreate(&e);
  if (cudaSuccess == r) *event_p = (void*)e;
  return xs_record_error(r, "cudaEventCreate");
}

double libxstream_b200_event_elapsed_ms(void* start, void* stop) {
  float ms = -1.f;
  if (NULL == start || NULL == stop) return -1.0;
  if (cudaSuccess != cudaEventSynchronize((cudaEvent_t)stop)) return -1.0;
  if (cudaSuccess != cudaEventElapsedTime(&ms, (cudaEvent_t)start, (cudaEvent_t)stop)) return -1.0;
  return (double)ms;
}

/* ------------------------------------------------------------------------- CUDA graphs */

int libxstream_b200_graph_begin(void* stream) {
  if (NULL == stream) return EXIT_FAILURE;
  if (EXIT_SUCCESS != xs_ensure_device()) return EXIT_FAILURE;
  return xs_record_error((int)cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal),
    "cudaStreamBeginCapture");
}

int libxstream_b200_graph_end(void* stream, void** graph_exec, int* nkernels) {
  cudaGraph_t graph = NULL;
  cudaGraphExec_t exec = NULL;
  size_t nnodes = 0, i;
  int r, count = 0;
  if (NULL == stream || NULL == graph_exec) return EXIT_FAILURE;
  *graph_exec = NULL;
  r = (int)cudaStreamEndCapture((cudaStream_t)stream, &graph);
  if (cudaSuccess != r) return xs_record_error(r, "cudaStreamEndCapture");
  if (NULL != nkernels && cudaSuccess == cudaGraphGetNodes(graph, NULL, &nnodes) && 0 < nnodes) {
    cudaGraphNode_t* const nodes = (cudaGraphNode_t*)malloc(sizeof(cudaGraphNode_t) * nnodes);
    if (NULL != nodes && cudaSuccess == cudaGraphGetNodes(graph, nodes, &nnodes)) {
      for (i = 0; i < nnodes; ++i) {
        enum cudaGraphNodeType type;
        if (cudaSuccess == cudaGraphNodeGetType(nodes[i], &type) && cudaGraphNodeTypeKernel == type) ++count;
      }
    }
    free(nodes);
  }
  if (NULL != nkernels) *nkernels = count;
  r = (int)cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (cudaSuccess != r) return xs_record_error(r, "cudaGraphInstantiate");
  *graph_exec = (void*)exec;
  return EXIT_SUCCESS;
}

int libxstream_b200_graph_launch(void* graph_exec, void* stream) {
  if (NULL == graph_exec) return EXIT_FAILURE;
  return xs_record_error((int)cudaGraphLaunch((cudaGraphExec_t)graph_exec, (cudaStream_t)stream), "cudaGraphLaunch");
}

int libxstream_b200_graph_destroy(void* graph_exec) {
  if (NULL == graph_exec) return EXIT_SUCCESS;
  return xs_record_error((int)cudaGraphExecDestroy((cudaGraphExec_t)graph_exec), "cudaGraphExecDestroy");
}
