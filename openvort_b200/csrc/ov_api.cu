// ov_api.cu - the C ABI of libov_gpu.so (include/openvort_b200.h): the
// reference's hot-path entry points over a host `struct tangle_state`, the
// run-time globals and boundary-image tables they read, and the ov_*
// extensions (device-resident state, point queries, error channel).
//
// Every reference-named call copies what it reads to the GPU, runs there and
// copies what it writes back before returning, so the reference's host code
// (reconnection, remeshing, frame output) sees the same tangle it would with
// its own functions.  No computation falls back to the CPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <cmath>
#include <mutex>
#include <string>

#include "openvort_b200.h"
#include "ov_internal.h"

// ======================================================================
// globals read by the hot path, with the reference's defaults
// (src/vortex_constants.c:24-95).  Default visibility: an executable that
// links the reference's vortex_constants.o interposes its own.
extern "C" {
double VORTEX_WIDTH = 1e-8;
double KAPPA = 9.97e-4;
int global_LIA_only = 0;
double global_alpha = 0.1;
double global_alpha_p = 0.01;
double global_dl_max = 5e-3;
int global_num_threads = 4;
int global_use_mutual_friction = 1;
int global_use_BH = 0;
double global_BH_resolution = 0.1;
int global_BH_quadtree = 0;
double global_BH_grain = 1e-8;
int global_hyperfriction = 1;
double global_max_curvature_scale = 0.2;
double global_hyperalpha = 0.5;
// loop removal (src/vortex_constants.c:48,65-74)
int global_small_loop_cutoff = 5;
int global_eliminate_origin_loops = 0;
double global_eliminate_loops_origin_cutoff = 3e-2;
int global_eliminate_zaxis_loops = 0;
double global_eliminate_loops_zaxis_cutoff = 2e-2;
int global_eliminate_outer_loops = 0;
double global_eliminate_outer_loops_cutoff = 1;
struct v_conf_t vn_conf;
struct v_conf_t vs_conf;
struct v_conf_t vb_conf;

// ----------------------------------------------------------------------
// boundary image tables: the same images in the same order as
// src/boundary_images.c:26-163 (a table of shifts that has to be alike for
// the image sums to agree).  wall_1_6 lists 5 images with n = 5 (the
// reference's n = 6 reads past its array).
static const struct image_tangle t_periodic_z_open_xy[] = {{{0, 0, -1}, -1}, {{0, 0, 1}, -1}};
static const struct image_tangle t_periodic_6[] = {{{-1, 0, 0}, -1}, {{0, -1, 0}, -1},
                                                   {{0, 0, -1}, -1}, {{0, 0, 1}, -1},
                                                   {{0, 1, 0}, -1},  {{1, 0, 0}, -1}};
static const struct image_tangle t_periodic_18[] = {
    {{-1, -1, 0}, -1}, {{-1, 0, -1}, -1}, {{-1, 0, 0}, -1}, {{-1, 0, 1}, -1}, {{-1, 1, 0}, -1},
    {{0, -1, -1}, -1}, {{0, -1, 0}, -1},  {{0, -1, 1}, -1}, {{0, 0, -1}, -1}, {{0, 0, 1}, -1},
    {{0, 1, -1}, -1},  {{0, 1, 0}, -1},   {{0, 1, 1}, -1},  {{1, -1, 0}, -1}, {{1, 0, -1}, -1},
    {{1, 0, 0}, -1},   {{1, 0, 1}, -1},   {{1, 1, 0}, -1}};
static const struct image_tangle t_periodic_26[] = {
    {{-1, -1, -1}, -1}, {{-1, -1, 0}, -1}, {{-1, -1, 1}, -1}, {{-1, 0, -1}, -1}, {{-1, 0, 0}, -1},
    {{-1, 0, 1}, -1},   {{-1, 1, -1}, -1}, {{-1, 1, 0}, -1},  {{-1, 1, 1}, -1},  {{0, -1, -1}, -1},
    {{0, -1, 0}, -1},   {{0, -1, 1}, -1},  {{0, 0, -1}, -1},  {{0, 0, 1}, -1},   {{0, 1, -1}, -1},
    {{0, 1, 0}, -1},    {{0, 1, 1}, -1},   {{1, -1, -1}, -1}, {{1, -1, 0}, -1},  {{1, -1, 1}, -1},
    {{1, 0, -1}, -1},   {{1, 0, 0}, -1},   {{1, 0, 1}, -1},   {{1, 1, -1}, -1},  {{1, 1, 0}, -1},
    {{1, 1, 1}, -1}};
static const struct image_tangle t_wall_2_4[] = {{{-1, 0, 0}, -1}, {{1, 0, 0}, -1},
                                                 {{0, -1, 0}, -1}, {{0, 1, 0}, -1},
                                                 {{0, 0, -1}, Z_L}, {{0, 0, 1}, Z_H}};
static const struct image_tangle t_wall_2_26[] = {
    {{-1, 0, 0}, -1},   {{1, 0, 0}, -1},    {{0, -1, 0}, -1},   {{0, 1, 0}, -1},
    {{-1, -1, 0}, -1},  {{-1, 1, 0}, -1},   {{1, -1, 0}, -1},   {{1, 1, 0}, -1},
    {{0, 0, -1}, Z_L},  {{1, 0, -1}, Z_L},  {{-1, 0, -1}, Z_L}, {{0, 1, -1}, Z_L},
    {{0, -1, -1}, Z_L}, {{1, 1, -1}, Z_L},  {{-1, 1, -1}, Z_L}, {{1, -1, -1}, Z_L},
    {{-1, -1, -1}, Z_L}, {{0, 0, 1}, Z_H},  {{1, 0, -1}, Z_H},  {{-1, 0, -1}, Z_H},
    {{0, 1, -1}, Z_H},  {{0, -1, -1}, Z_H}, {{1, 1, -1}, Z_H},  {{-1, 1, -1}, Z_H},
    {{1, -1, -1}, Z_H}, {{-1, -1, -1}, Z_H}};
static const struct image_tangle t_wall_2_2[] = {{{-1, 0, 0}, -1}, {{1, 0, 0}, -1},
                                                 {{0, -1, 0}, Y_L}, {{0, 1, 0}, Y_H},
                                                 {{0, 0, -1}, Z_L}, {{0, 0, 1}, Z_H}};
static const struct image_tangle t_wall_1_open[] = {{{0, 0, -1}, Z_L}};
static const struct image_tangle t_wall_1_6[] = {{{-1, 0, 0}, -1}, {{0, -1, 0}, -1},
                                                 {{0, 0, -1}, Z_L}, {{0, 1, 0}, -1},
                                                 {{1, 0, 0}, -1}};
static const struct image_tangle t_wall_1_18[] = {
    {{-1, -1, 0}, -1}, {{-1, 0, -1}, Z_L}, {{-1, 0, 0}, -1}, {{-1, 0, 1}, -1}, {{-1, 1, 0}, -1},
    {{0, -1, -1}, Z_L}, {{0, -1, 0}, -1},  {{0, -1, 1}, -1}, {{0, 0, -1}, Z_L}, {{0, 0, 1}, -1},
    {{0, 1, -1}, Z_L},  {{0, 1, 0}, -1},   {{0, 1, 1}, -1},  {{1, -1, 0}, -1},  {{1, 0, -1}, Z_L},
    {{1, 0, 0}, -1},    {{1, 0, 1}, -1},   {{1, 1, 0}, -1}};
static const struct image_tangle t_wall_1_26[] = {
    {{-1, -1, -1}, Z_L}, {{-1, -1, 0}, -1}, {{-1, -1, 1}, -1}, {{-1, 0, -1}, Z_L}, {{-1, 0, 0}, -1},
    {{-1, 0, 1}, -1},    {{-1, 1, -1}, Z_L}, {{-1, 1, 0}, -1},  {{-1, 1, 1}, -1},  {{0, -1, -1}, Z_L},
    {{0, -1, 0}, -1},    {{0, -1, 1}, -1},  {{0, 0, -1}, Z_L},  {{0, 0, 1}, -1},   {{0, 1, -1}, Z_L},
    {{0, 1, 0}, -1},     {{0, 1, 1}, -1},   {{1, -1, -1}, Z_L}, {{1, -1, 0}, -1},  {{1, -1, 1}, -1},
    {{1, 0, -1}, Z_L},   {{1, 0, 0}, -1},   {{1, 0, 1}, -1},   {{1, 1, -1}, Z_L},  {{1, 1, 0}, -1},
    {{1, 1, 1}, -1}};
// the reference's channel_z lists {0,0,1} twice and no {0,0,-1}
static const struct image_tangle t_channel_z[] = {{{-1, 0, 0}, X_L}, {{1, 0, 0}, X_H},
                                                  {{0, -1, 0}, Y_L}, {{0, 1, 0}, Y_H},
                                                  {{0, 0, 1}, -1},   {{0, 0, 1}, -1}};

const struct boundary_images open_boundaries = {NULL, 0};
const struct boundary_images periodic_z_open_xy = {t_periodic_z_open_xy, 2};
const struct boundary_images periodic_6 = {t_periodic_6, 6};
const struct boundary_images periodic_18 = {t_periodic_18, 18};
const struct boundary_images periodic_26 = {t_periodic_26, 26};
const struct boundary_images wall_1_open = {t_wall_1_open, 1};
const struct boundary_images wall_1_6 = {t_wall_1_6, 5};
const struct boundary_images wall_1_18 = {t_wall_1_18, 18};
const struct boundary_images wall_1_26 = {t_wall_1_26, 26};
const struct boundary_images wall_2_4 = {t_wall_2_4, 6};
const struct boundary_images wall_2_2 = {t_wall_2_2, 6};
// the reference's wall_2_26 has n = 6 over its 26 entries; kept
const struct boundary_images wall_2_26 = {t_wall_2_26, 6};
const struct boundary_images channel_z = {t_channel_z, 6};
}  // extern "C"

// ======================================================================
// errors, buffers, statistics

namespace {
thread_local int tl_err = OV_OK;
thread_local char tl_msg[512] = "";
thread_local OvStatsAcc tl_stats = {0, 0, 0, 0, 0, 0, 0};
thread_local ov_state_impl* tl_last_state = nullptr;
int g_precision = OV_PREC_FP64;
int g_rk4_classic = 0;
// FP64 near field of the mixed form, in units of global_dl_max: at 8 (and
// at 4 or 16) the mixed velocities stay within ~3e-6 of the FP64 ones on the
// benchmark tangles
double g_near_factor = 8.0;
double g_col_cut = 1e-8;   // the reference's colinearity cut-off (src/tangle.c:505)
int g_device = -1;
std::mutex g_init_mutex;
}  // namespace

void ov_set_error(int code, const char* fmt, ...) {
  tl_err = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(tl_msg, sizeof(tl_msg), fmt, ap);
  va_end(ap);
  if (!getenv("OV_QUIET")) fprintf(stderr, "libov_gpu: error %d: %s\n", code, tl_msg);
  const char* ab = getenv("OV_ABORT_ON_ERROR");
  if (ab && ab[0] == '1') abort();
}

bool ov_cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  ov_set_error(e == cudaErrorMemoryAllocation ? OV_ERR_NOMEM : OV_ERR_CUDA, "%s: %s", what,
               cudaGetErrorString(e));
  return false;
}

bool DevBuf::reserve(size_t n) {
  if (n <= bytes && p) return true;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  size_t want = n + n / 4 + 256;   // headroom so slowly growing tangles rarely reallocate
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    ov_cuda_ok(e, "cudaMalloc");
    return false;
  }
  bytes = want;
  return true;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

OvStatsAcc& ov_stats_tls() { return tl_stats; }

static std::atomic<long long> g_launches{0};
void ov_note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long ov_launches() { return g_launches.load(std::memory_order_relaxed); }

extern "C" {

int ov_last_error(void) { return tl_err; }
const char* ov_last_error_message(void) { return tl_msg; }
void ov_clear_error(void) {
  tl_err = OV_OK;
  tl_msg[0] = 0;
}
const char* ov_error_string(int code) {
  switch (code) {
    case OV_OK: return "ok";
    case OV_ERR_NO_DEVICE: return "no usable CUDA device (sm_100a required)";
    case OV_ERR_CUDA: return "CUDA runtime error";
    case OV_ERR_INVALID: return "invalid argument or tangle";
    case OV_ERR_NONFINITE: return "non-finite value";
    case OV_ERR_FLOW: return "unknown external flow or missing flow parameter";
    case OV_ERR_TREE_DEPTH: return "octree deeper than 32 levels";
    case OV_ERR_TIMEOUT: return "bounded device wait ran out";
    case OV_ERR_NOMEM: return "device out of memory";
    default: return "unknown error";
  }
}

void ov_set_precision(int mode) { g_precision = mode == OV_PREC_MIXED ? OV_PREC_MIXED : OV_PREC_FP64; }
int ov_get_precision(void) { return g_precision; }
void ov_set_rk4_classic(int classic) { g_rk4_classic = classic ? 1 : 0; }
void ov_set_mixed_near_factor(double f) { g_near_factor = f > 0 ? f : 0; }
double ov_get_mixed_near_factor(void) { return g_near_factor; }
void ov_set_colinear_cutoff(double eps) { g_col_cut = eps > 0 ? eps : 0; }
double ov_get_colinear_cutoff(void) { return g_col_cut; }
int ov_get_rk4_classic(void) { return g_rk4_classic; }

int ov_init(int device) {
  std::lock_guard<std::mutex> lk(g_init_mutex);
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    ov_set_error(OV_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    return OV_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= n) device = 0;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
    ov_set_error(OV_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a", device,
                 prop.major, prop.minor);
    return OV_ERR_NO_DEVICE;
  }
  if (!ov_cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return tl_err;
  g_device = device;
  return OV_OK;
}

}  // extern "C"

static bool ensure_init() {
  if (g_device >= 0) {
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != g_device) cudaSetDevice(g_device);
    return true;
  }
  return ov_init(0) == OV_OK;
}

// ======================================================================
// parameter capture

namespace {

struct FlowSpec {
  const char* name;
  int kind;
  const char* scalars[4];
  const char* vectors[2];
  int n_required_scalars;
};

// parameter names per flow, in the reference's v_confs[] order
// (src/external_velocity.c:85-170)
const FlowSpec kFlows[] = {
    {"no flow", OVF_NONE, {0}, {0}, 0},
    {"spherical", OVF_SPHERICAL, {"strength", "cutoff"}, {0}, 2},
    {"simple", OVF_SIMPLE, {0}, {"external_v"}, 0},
    {"spherical and simple", OVF_SPHERICAL_SIMPLE, {"strength", "cutoff"}, {"external_v"}, 2},
    {"cylindrical", OVF_CYLINDRICAL, {"strength", "cutoff"}, {0}, 2},
    {"oscillating", OVF_OSCILLATING, {"strength", "frequency"}, {"wave", "polarization"}, 2},
    {"oscillating slit", OVF_OSCILLATING_SLIT, {"strength", "frequency", "cutoff"}, {0}, 3},
    {"coscos", OVF_COSCOS, {"k", "v0", "l"}, {0}, 3},
    {"coscos-divfree", OVF_COSCOS_DIVFREE, {"k", "v0", "l"}, {0}, 3},
    {"cos-divfree", OVF_COS_DIVFREE, {"k", "v0", "l"}, {0}, 3},
    {"simple-shear", OVF_SIMPLE_SHEAR, {"rate", "v0"}, {0}, 2},
    {"rotosc", OVF_ROTOSC, {"freq", "amp"}, {0}, 2},
    {"DG", OVF_DG, {"rot", "vz"}, {0}, 2},
    {"rotosc-boundary", OVF_ROTOSC_BOUNDARY, {"freq", "amp"}, {0}, 2},
    {"constant acceleration", OVF_CONST_ACCEL, {"accel"}, {0}, 1},
    {"parabolic", OVF_PARABOLIC, {"H", "amp"}, {0}, 2},
};

const v_param_t* find_param(const v_conf_t& c, const char* name) {
  for (int k = 0; k < c.n_params && k < 32; ++k)
    if (c.v_params[k].name && strcmp(c.v_params[k].name, name) == 0) return &c.v_params[k];
  return nullptr;
}

bool parse_flow(const v_conf_t& c, const char* which, OvFlow& f) {
  memset(&f, 0, sizeof(f));
  if (!c.name) {
    ov_set_error(OV_ERR_FLOW, "%s is not configured (no flow name)", which);
    return false;
  }
  for (const FlowSpec& s : kFlows) {
    if (strcmp(s.name, c.name) != 0) continue;
    f.kind = s.kind;
    for (int i = 0; i < 4 && s.scalars[i]; ++i) {
      const v_param_t* p = find_param(c, s.scalars[i]);
      if (!p) {
        ov_set_error(OV_ERR_FLOW, "%s flow '%s' lacks parameter '%s'", which, c.name, s.scalars[i]);
        return false;
      }
      f.s[i] = p->value.scalar;
    }
    for (int i = 0; i < 2 && s.vectors[i]; ++i) {
      const v_param_t* p = find_param(c, s.vectors[i]);
      if (!p) {
        ov_set_error(OV_ERR_FLOW, "%s flow '%s' lacks parameter '%s'", which, c.name, s.vectors[i]);
        return false;
      }
      for (int a = 0; a < 3; ++a) f.v[i][a] = p->value.vector.p[a];
    }
    return true;
  }
  ov_set_error(OV_ERR_FLOW, "%s: unknown flow '%s'", which, c.name);
  return false;
}

bool any_pinned(const tangle_state* t) {
  for (int k = 0; k < t->N; ++k)
    if (t->status[k].status == PINNED) return true;
  return false;
}

// Everything the kernels read from the globals and the tangle header.
bool capture_params(const tangle_state* t, OvParams& P, bool need_flows) {
  memset(&P, 0, sizeof(P));
  P.kappa = KAPPA;
  P.core_a = VORTEX_WIDTH;
  P.f4pi = KAPPA / 4 / M_PI;
  for (int c = 0; c < 3; ++c) {
    P.lo[c] = t->box.bottom_left_back.p[c];
    P.hi[c] = t->box.top_right_front.p[c];
    P.L[c] = P.hi[c] - P.lo[c];
    P.periodic[c] = t->box.wall[2 * c] == WALL_PERIODIC;
  }
  if (t->bimg.n < 0 || t->bimg.n > OV_MAX_IMAGES || (t->bimg.n > 0 && !t->bimg.images)) {
    ov_set_error(OV_ERR_INVALID, "boundary image table with %d images (max %d)", t->bimg.n,
                 OV_MAX_IMAGES);
    return false;
  }
  P.n_img = t->bimg.n;
  for (int j = 0; j < P.n_img; ++j) {
    for (int c = 0; c < 3; ++c) P.img[j][c] = t->bimg.images[j].shift[c];
    P.img[j][3] = t->bimg.images[j].reflect;
    if (P.img[j][3] < -1 || P.img[j][3] > 5) {
      ov_set_error(OV_ERR_INVALID, "image %d reflects in face %d", j, P.img[j][3]);
      return false;
    }
  }
  P.lia_only = global_LIA_only;
  P.use_bh = global_use_BH;
  P.quadtree = global_BH_quadtree;
  P.use_mf = global_use_mutual_friction;
  P.hyperfriction = global_hyperfriction;
  P.precision = g_precision;
  P.theta = global_BH_resolution;
  P.grain = global_BH_grain;
  P.dl_max = global_dl_max;
  P.near2 = (g_near_factor * global_dl_max) * (g_near_factor * global_dl_max);
  P.alpha = global_alpha;
  P.alpha_p = global_alpha_p;
  P.max_curv = global_max_curvature_scale;
  P.hyperalpha = global_hyperalpha;
  P.col_cut = g_col_cut;
  if (need_flows) {
    if (!parse_flow(vs_conf, "vs_conf", P.vs)) return false;
    if (P.use_mf && !parse_flow(vn_conf, "vn_conf", P.vn)) return false;
    if (any_pinned(t) && !parse_flow(vb_conf, "vb_conf", P.vb)) return false;
  }
  return true;
}

}  // namespace

// Box, image table and globals of a tangle header (no flows, no node arrays
// read): the parameters of a point query.
bool ov_capture_header_params(const struct tangle_state* t, OvParams& P) {
  return capture_params(t, P, false);
}

// Box, image table, globals and flows of a tangle (the pinned-node scan of
// the boundary flow covers the tangle's N slots).
bool ov_capture_params(const tangle_state* t, OvParams& P) { return capture_params(t, P, true); }

// ======================================================================
// state management

bool ov_state_reserve(ov_state_impl* s, int n) {
  if (!s->stream) {
    OV_TRY_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    OV_TRY_CUDA(cudaEventCreate(&s->ev0));
    OV_TRY_CUDA(cudaEventCreate(&s->ev1));
    OV_TRY_CUDA(cudaEventCreate(&s->ev2));
    if (!s->dflag.reserve(64)) return false;
  }
  s->n = n;
  if (n <= s->cap) return true;
  size_t v3 = sizeof(double) * 3 * (size_t)n, sc = sizeof(double) * (size_t)n;
  DevBuf* vecs[] = {&s->pos, &s->tan, &s->nrm, &s->vels, &s->vs, &s->pos0, &s->spos, &s->stan,
                    &s->snrm, &s->svs, &s->k2, &s->k3, &s->k4, &s->v_nl, &s->v_img};
  for (DevBuf* b : vecs)
    if (!b->reserve(v3)) return false;
  if (!s->dxi.reserve(sc) || !s->sdxi.reserve(sc)) return false;
  if (!s->links.reserve(sizeof(int2) * (size_t)n) || !s->status.reserve(sizeof(int2) * (size_t)n))
    return false;
  s->cap = n;
  return true;
}

static void state_release(ov_state_impl* s) {
  ov_frames_release(s);
  DevBuf* bufs[] = {&s->pos, &s->links, &s->status, &s->dxi, &s->tan, &s->nrm, &s->vels, &s->vs,
                    &s->pos0, &s->spos, &s->sdxi, &s->stan, &s->snrm, &s->svs, &s->k2, &s->k3,
                    &s->k4, &s->v_nl, &s->v_img, &s->img_part, &s->seg64, &s->segid, &s->dflag,
                    &s->xown};
  for (DevBuf* b : bufs) b->release();
  ov_tree_release(&s->tree);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->ev2) cudaEventDestroy(s->ev2);
  s->stream = nullptr;
  s->cap = s->n = 0;
}

// The link and status arrays of struct tangle_state are pairs of ints
// (struct neighbour_t, node_status), copied as int2.
static_assert(sizeof(struct neighbour_t) == 8, "neighbour_t layout");
static_assert(sizeof(node_status) == 8, "node_status layout");
static_assert(sizeof(struct vec3d) == 24, "vec3d layout");

static bool upload(ov_state_impl* s, const void* host, DevBuf& dev, size_t bytes) {
  if (!host) {
    ov_set_error(OV_ERR_INVALID, "tangle array missing");
    return false;
  }
  OV_TRY_CUDA(cudaMemcpyAsync(dev.p, host, bytes, cudaMemcpyHostToDevice, s->stream));
  return true;
}

static bool download(ov_state_impl* s, void* host, const DevBuf& dev, size_t bytes) {
  if (!host) return true;
  OV_TRY_CUDA(cudaMemcpyAsync(host, dev.p, bytes, cudaMemcpyDeviceToHost, s->stream));
  return true;
}

// Copy the tangle's node structure and positions in.
static bool upload_tangle(ov_state_impl* s, const tangle_state* t, bool need_flows) {
  if (!t || t->N < 0) {
    ov_set_error(OV_ERR_INVALID, "null tangle");
    return false;
  }
  size_t n = (size_t)t->N;
  // targets (non-EMPTY, non-PINNED) and segments (forward link) for the
  // interaction counts of the direct sum
  // and a check that every link and wall index the kernels follow is in
  // range, so a malformed tangle is an error instead of a stray device read
  int nt = 0, ns = 0, na = 0;
  if (t->N > 0 && (!t->status || !t->connections || !t->vnodes)) {
    ov_set_error(OV_ERR_INVALID, "tangle without status, connection or position arrays");
    return false;
  }
  for (int k = 0; k < t->N; ++k) {
    int st = t->status[k].status;
    if (st == EMPTY) continue;
    int f = t->connections[k].forward, r = t->connections[k].reverse;
    if (st < EMPTY || st > PINNED_SLIP || f < -1 || f >= t->N || r < -1 || r >= t->N ||
        (f >= 0 && t->status[f].status == EMPTY) || (r >= 0 && t->status[r].status == EMPTY) ||
        ((st == PINNED || st == PINNED_SLIP) &&
         (t->status[k].pin_wall < 0 || t->status[k].pin_wall > 5))) {
      ov_set_error(OV_ERR_INVALID, "node %d: status %d, links (%d, %d), wall %d out of range", k, st,
                   f, r, (int)t->status[k].pin_wall);
      return false;
    }
    // a NaN or infinite position of a live node is refused here, before any
    // launch, so no output array is written (EMPTY slots may hold anything)
    const vec3d& x = t->vnodes[k];
    if (!(std::isfinite(x.p[0]) && std::isfinite(x.p[1]) && std::isfinite(x.p[2]))) {
      ov_set_error(OV_ERR_NONFINITE, "node %d: non-finite position (%g, %g, %g)", k, x.p[0], x.p[1],
                   x.p[2]);
      return false;
    }
    ++na;
    if (st != PINNED) ++nt;
    if (f >= 0) ++ns;
  }
  // the host arrays are valid: now the device
  if (!ensure_init()) return false;
  if (!capture_params(t, s->P, need_flows)) return false;
  if (!ov_state_reserve(s, t->N)) return false;
  s->n_targets = nt;
  s->n_segments = ns;
  s->n_active = na;
  for (int f = 0; f < 6; ++f) s->walls[f] = t->box.wall[f];
  if (n == 0) return true;
  return upload(s, t->vnodes, s->pos, 24 * n) && upload(s, t->connections, s->links, 8 * n) &&
         upload(s, t->status, s->status, 8 * n);
}

static bool sync(ov_state_impl* s) {
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return true;
}

bool ov_ensure_init() { return ensure_init(); }

bool ov_upload_tangle(ov_state_impl* s, const tangle_state* t) { return upload_tangle(s, t, true); }

bool ov_download_fields(ov_state_impl* s, tangle_state* t, int what) {
  if (t->N != s->n) {
    ov_set_error(OV_ERR_INVALID, "tangle has %d slots, state %d", t->N, s->n);
    return false;
  }
  size_t n = (size_t)s->n;
  if (n == 0) return true;
  bool ok = true;
  if (what & OV_FIELD_POS) ok = ok && download(s, t->vnodes, s->pos, 24 * n);
  if (what & OV_FIELD_VELS) ok = ok && download(s, t->vels, s->vels, 24 * n);
  if (what & OV_FIELD_VS) ok = ok && download(s, t->vs, s->vs, 24 * n);
  if (what & OV_FIELD_TANGENTS) ok = ok && download(s, t->tangents, s->tan, 24 * n);
  if (what & OV_FIELD_NORMALS) ok = ok && download(s, t->normals, s->nrm, 24 * n);
  if (what & OV_FIELD_DXI) ok = ok && download(s, t->dxi, s->dxi, 8 * n);
  return ok && sync(s);
}

// The Biot-Savart sums of an evaluation into v_nl, v_img: the tree build and
// walk (for the targets at key positions [k0, k0 + k_count) of the tree; all
// of them when k_count < 0), or the direct sum.
static bool bs_sums(ov_state_impl* s, const double* pos, OvTree* external_tree, int k0, int k_count) {
  tl_last_state = s;
  tl_stats = OvStatsAcc{0, 0, 0, 0, 0, 0, 0};
  cudaEventRecord(s->ev0, s->stream);
  cudaEventRecord(s->ev1, s->stream);
  cudaEventRecord(s->ev2, s->stream);
  double* v_nl = s->v_nl.as<double>();
  double* v_img = s->v_img.as<double>();
  if (!s->P.lia_only) {
    if (s->P.use_bh) {
      OvTree* tree = external_tree;
      if (!tree) {
        if (!ov_tree_build(s, pos, &s->tree)) return false;
        tree = &s->tree;
      }
      if (!ov_tree_walk_nodes(s, tree, pos, tree == &s->tree, v_nl, v_img, k0, k_count)) return false;
    } else {
      if (!ov_direct_nodes(s, pos, v_nl, v_img)) return false;
      // every target against every segment, per image (src/tangle.c:612-636)
      tl_stats.interactions = (double)s->n_targets * (double)s->n_segments * (1 + s->P.n_img);
    }
  }
  return true;
}

// The epilogue of an evaluation over every node, and the state's counters.
static bool finish_velocities(ov_state_impl* s, double t, const double* pos, const double* tan,
                              const double* nrm, double* vels, double* vs) {
  if (!ov_epilogue(s, t, pos, tan, nrm, s->v_nl.as<double>(), s->v_img.as<double>(), vels, vs, 0, s->n))
    return false;
  // the epilogue synchronised the stream: fold this evaluation into the
  // state's counters (device times from the events around the tree build and
  // the Biot-Savart kernel)
  float build_ms = 0, bs_ms = 0;
  cudaEventElapsedTime(&build_ms, s->ev0, s->ev1);
  cudaEventElapsedTime(&bs_ms, s->ev1, s->ev2);
  tl_stats.build_ms = build_ms;
  tl_stats.eval_ms = bs_ms;
  tl_stats.total_ms = build_ms + bs_ms;
  s->acc_evals += 1;
  s->acc_build_ms += build_ms;
  s->acc_bs_ms += bs_ms;
  s->acc_bs_launches += s->P.lia_only ? 0 : 1;
  s->acc_inter += tl_stats.interactions;
  s->acc_cells += tl_stats.cell_interactions;
  s->acc_warp_iter += tl_stats.warp_iterations;
  return true;
}

bool ov_velocities(ov_state_impl* s, double t, const double* pos, const double* dxi,
                   const double* tan, const double* nrm, double* vels, double* vs,
                   OvTree* external_tree) {
  (void)dxi;
  return bs_sums(s, pos, external_tree, 0, -1) && finish_velocities(s, t, pos, tan, nrm, vels, vs);
}

// ======================================================================
// ov_state API

struct ov_state {
  ov_state_impl impl;
};

ov_state_impl* ov_state_impl_of(ov_state* s) { return &s->impl; }

extern "C" {

ov_state* ov_state_create(void) {
  if (!ensure_init()) return nullptr;
  return new ov_state();
}

void ov_state_destroy(ov_state* s) {
  if (!s) return;
  state_release(&s->impl);
  delete s;
}

int ov_state_upload(ov_state* st, const struct tangle_state* t) {
  ov_clear_error();
  if (!st) { ov_set_error(OV_ERR_INVALID, "null state"); return tl_err; }
  ov_state_impl* s = &st->impl;
  if (!upload_tangle(s, t, true)) return tl_err;
  size_t n = (size_t)t->N;
  if (n && t->vels && !upload(s, t->vels, s->vels, 24 * n)) return tl_err;
  if (!sync(s)) return tl_err;
  return OV_OK;
}

int ov_state_download(ov_state* st, struct tangle_state* t, int what) {
  ov_clear_error();
  if (!st || !t) { ov_set_error(OV_ERR_INVALID, "null state or tangle"); return tl_err; }
  if (!ov_download_fields(&st->impl, t, what)) return tl_err;
  return OV_OK;
}

int ov_state_update_tangle(ov_state* st, double t) {
  ov_clear_error();
  ov_state_impl* s = &st->impl;
  s->P.precision = g_precision;
  if (!ov_geometry(s, s->pos.as<double>(), s->dxi.as<double>(), s->tan.as<double>(),
                   s->nrm.as<double>()))
    return tl_err;
  if (!ov_velocities(s, t, s->pos.as<double>(), s->dxi.as<double>(), s->tan.as<double>(),
                     s->nrm.as<double>(), s->vels.as<double>(), s->vs.as<double>(), nullptr))
    return tl_err;
  return OV_OK;
}

int ov_state_rk4_step(ov_state* st, double t, double dt) {
  ov_clear_error();
  ov_state_impl* s = &st->impl;
  s->P.precision = g_precision;
  if (!ov_rk4(s, t, dt, g_rk4_classic)) return tl_err;
  return OV_OK;
}

int ov_state_run(ov_state* st, double t0, double dt, int nsteps) {
  ov_clear_error();
  ov_state_impl* s = &st->impl;
  if (!s->ev_run0) {
    cudaEventCreate(&s->ev_run0);
    cudaEventCreate(&s->ev_run1);
  }
  cudaEventRecord(s->ev_run0, s->stream);
  double t = t0;
  for (int i = 0; i < nsteps; ++i) {
    int e = ov_state_update_tangle(st, t);
    if (e) return e;
    e = ov_state_rk4_step(st, t, dt);
    if (e) return e;
    t += dt;
  }
  cudaEventRecord(s->ev_run1, s->stream);
  if (!sync(s)) return tl_err;
  float ms = 0;
  cudaEventElapsedTime(&ms, s->ev_run0, s->ev_run1);
  s->last_run_ms = ms;
  return OV_OK;
}

// ---------------------------------------------------------------- shards
// Key positions per rank: c = ceil(active nodes / world); rank r holds
// [r c, min((r + 1) c, active)).
static int shard_chunk(const ov_state_impl* s, int world) {
  return world > 0 ? (s->n_active + world - 1) / world : 0;
}

size_t ov_state_shard_bytes(ov_state* st, int world) {
  if (!st || world < 1) return 0;
  return sizeof(double) * 6 * (size_t)shard_chunk(&st->impl, world) * (size_t)world;
}

int ov_state_shard(ov_state* st, int rank, int world, void* xbuf, size_t bytes) {
  ov_clear_error();
  if (!st || world < 1 || rank < 0 || rank >= world) {
    ov_set_error(OV_ERR_INVALID, "ov_state_shard: rank %d of %d", rank, world);
    return tl_err;
  }
  ov_state_impl* s = &st->impl;
  const size_t need = ov_state_shard_bytes(st, world);
  if (!xbuf && world > 1) {
    ov_set_error(OV_ERR_INVALID, "ov_state_shard: %d ranks need an exchange buffer", world);
    return tl_err;
  }
  if (xbuf && (bytes < need || (reinterpret_cast<uintptr_t>(xbuf) & 7) != 0)) {
    ov_set_error(OV_ERR_INVALID, "ov_state_shard: exchange buffer of %zu bytes at %p, need %zu, 8-aligned",
                 bytes, xbuf, need);
    return tl_err;
  }
  if (!xbuf) {
    if (!s->xown.reserve(need > 0 ? need : 8)) return tl_err;
    xbuf = s->xown.p;
    bytes = s->xown.bytes;
  }
  s->shard_rank = rank;
  s->shard_world = world;
  s->xbuf = static_cast<double*>(xbuf);
  s->xbytes = bytes;
  return OV_OK;
}

// positions, geometry and outputs of stage q: 0 = update_tangle at the
// positions, 1..3 = the stages of rk4_step2 (src/vortex_dynamics.c:76-92)
struct ShardStage {
  const double* pos;
  double *dxi, *tan, *nrm, *vels, *vs;
  double t;
};

static ShardStage shard_stage(ov_state_impl* s, int q, double t, double dt) {
  if (q == 0)
    return {s->pos.as<double>(), s->dxi.as<double>(), s->tan.as<double>(), s->nrm.as<double>(),
            s->vels.as<double>(), s->vs.as<double>(), t};
  double* ks[3] = {s->k2.as<double>(), s->k3.as<double>(), s->k4.as<double>()};
  return {s->spos.as<double>(), s->sdxi.as<double>(), s->stan.as<double>(), s->snrm.as<double>(),
          ks[q - 1], s->svs.as<double>(), q < 3 ? t + dt / 2 : t + dt};
}

static bool shard_ready(ov_state_impl* s, int q) {
  if (q < 0 || q > 3) {
    ov_set_error(OV_ERR_INVALID, "shard stage %d (0..3)", q);
    return false;
  }
  if (!s->xbuf || s->xbytes < sizeof(double) * 6 * (size_t)shard_chunk(s, s->shard_world) * s->shard_world) {
    ov_set_error(OV_ERR_INVALID, "no exchange buffer for %d active nodes: call ov_state_shard after the upload",
                 s->n_active);
    return false;
  }
  if (!s->P.lia_only && !s->P.use_bh) {
    ov_set_error(OV_ERR_INVALID, "sharded evaluations need the Barnes-Hut path (global_use_BH)");
    return false;
  }
  return true;
}

int ov_state_shard_begin(ov_state* st, int q, double t, double dt) {
  ov_clear_error();
  if (!st) { ov_set_error(OV_ERR_INVALID, "null state"); return tl_err; }
  ov_state_impl* s = &st->impl;
  s->P.precision = g_precision;
  if (!shard_ready(s, q)) return tl_err;
  if (q > 0 && !ov_rk4_stage_positions(s, q, dt, g_rk4_classic)) return tl_err;
  const ShardStage g = shard_stage(s, q, t, dt);
  if (!ov_geometry(s, g.pos, g.dxi, g.tan, g.nrm)) return tl_err;
  const int c = shard_chunk(s, s->shard_world);
  if (!bs_sums(s, g.pos, nullptr, s->shard_rank * c, c)) return tl_err;
  s->shard_inter = tl_stats.interactions;
  s->shard_cells = tl_stats.cell_interactions;
  s->shard_warp_iter = tl_stats.warp_iterations;
  if (!s->P.lia_only && !ov_shard_pack(s, s->shard_rank * c, c, s->xbuf, s->xbytes / sizeof(double)))
    return tl_err;
  // the caller's exchange reads xbuf from another stream
  if (!sync(s)) return tl_err;
  return OV_OK;
}

int ov_state_shard_end(ov_state* st, int q, double t, double dt) {
  ov_clear_error();
  if (!st) { ov_set_error(OV_ERR_INVALID, "null state"); return tl_err; }
  ov_state_impl* s = &st->impl;
  if (!shard_ready(s, q)) return tl_err;
  const ShardStage g = shard_stage(s, q, t, dt);
  if (!s->P.lia_only && !ov_shard_unpack(s, s->xbuf, s->xbytes / sizeof(double))) return tl_err;
  tl_last_state = s;
  tl_stats = OvStatsAcc{s->shard_inter, s->shard_cells, 0, 0, 0, 0, s->shard_warp_iter};
  if (!finish_velocities(s, g.t, g.pos, g.tan, g.nrm, g.vels, g.vs)) return tl_err;
  if (q == 3 && !(ov_rk4_combine(s, dt) && sync(s))) return tl_err;
  return OV_OK;
}

int ov_state_get_stats(ov_state* st, ov_run_stats* out) {
  if (!st || !out) return OV_ERR_INVALID;
  ov_state_impl* s = &st->impl;
  out->evals = s->acc_evals;
  out->interactions = s->acc_inter;
  out->cell_interactions = s->acc_cells;
  out->bs_kernel_ms = s->acc_bs_ms;
  out->bs_launches = s->acc_bs_launches;
  out->build_ms = s->acc_build_ms;
  out->last_run_ms = s->last_run_ms;
  out->launches = (double)(ov_launches() - s->launches_at_reset);
  out->n_targets = s->n_targets;
  out->n_segments = s->n_segments;
  out->warp_iterations = s->acc_warp_iter;
  return OV_OK;
}

void ov_state_reset_stats(ov_state* st) {
  if (!st) return;
  ov_state_impl* s = &st->impl;
  s->acc_evals = s->acc_inter = s->acc_cells = s->acc_bs_ms = s->acc_bs_launches = 0;
  s->acc_warp_iter = 0;
  s->acc_build_ms = 0;
  s->launches_at_reset = ov_launches();
}

int ov_state_eval_points(ov_state* st, int npts, const double* pts, const int* skip, int method,
                         double* out) {
  ov_clear_error();
  ov_state_impl* s = &st->impl;
  s->P.precision = g_precision;
  if (npts <= 0) return OV_OK;
  DevBuf dp, ds, dout;
  if (!dp.reserve(sizeof(double) * 3 * npts) || !dout.reserve(sizeof(double) * 3 * npts)) return tl_err;
  if (skip && !ds.reserve(sizeof(int) * npts)) return tl_err;
  DevBuf dimg;
  if (!dimg.reserve(sizeof(double) * 3 * npts)) return tl_err;
  bool ok = upload(s, pts, dp, sizeof(double) * 3 * npts);
  if (ok && skip) ok = upload(s, skip, ds, sizeof(int) * npts);
  if (ok) {
    const int* dsk = skip ? ds.as<int>() : nullptr;
    if (method == 1) {
      ok = ov_tree_build(s, s->pos.as<double>(), &s->tree) &&
           ov_tree_walk_points(s, &s->tree, npts, dp.as<double>(), dsk, s->P.theta,
                               dout.as<double>(), dimg.as<double>());
    } else {
      ok = ov_direct_points(s, s->pos.as<double>(), npts, dp.as<double>(), dsk, nullptr, 0,
                            dout.as<double>(), dimg.as<double>());
    }
    ok = ok && ov_add3(s->stream, dout.as<double>(), dimg.as<double>(), dout.as<double>(), npts);
  }
  ok = ok && download(s, out, dout, sizeof(double) * 3 * npts) && sync(s);
  dp.release();
  ds.release();
  dout.release();
  dimg.release();
  return ok ? OV_OK : tl_err;
}

int ov_get_last_stats(ov_eval_stats* out) {
  if (!out) return OV_ERR_INVALID;
  memset(out, 0, sizeof(*out));
  ov_state_impl* s = tl_last_state;
  out->interactions = tl_stats.interactions;
  out->cell_interactions = tl_stats.cell_interactions;
  out->cells = tl_stats.cells;
  if (s && s->stream) {
    cudaStreamSynchronize(s->stream);
    float a = 0, b = 0;
    if (cudaEventElapsedTime(&a, s->ev0, s->ev1) == cudaSuccess) out->build_ms = a;
    if (cudaEventElapsedTime(&b, s->ev1, s->ev2) == cudaSuccess) out->eval_ms = b;
    // an event not recorded yet fails the query above; drop that error so
    // it is not reported by the next launch check
    (void)cudaGetLastError();
    out->total_ms = out->build_ms + out->eval_ms;
  }
  return OV_OK;
}

}  // extern "C"

// ======================================================================
// reference-named entry points over host tangles

namespace {
// One device state per host thread for the reference-named calls.
ov_state_impl& tls_state() {
  thread_local ov_state_impl* s = nullptr;
  if (!s) s = new ov_state_impl();
  return *s;
}

// The device-side tree behind an opaque struct octree*.
struct TreeHandle {
  ov_state_impl st;   // its own node snapshot, stream and buffers
};
}  // namespace

struct octree {
  TreeHandle h;
};

extern "C" {

struct vec3d shifted(const struct image_tangle* shift, const struct tangle_state* tangle,
                     const struct vec3d* r) {
  // host arithmetic on one point (src/tangle.c:39-79); not a kernel
  struct vec3d rs = *r;
  for (int k = 0; k < 3; ++k) {
    double L = tangle->box.top_right_front.p[k] - tangle->box.bottom_left_back.p[k];
    rs.p[k] -= L * shift->shift[k];
  }
  int f = shift->reflect;
  if (f >= 0 && f < 6) {
    int c = f / 2;
    double w = (f % 2 == 0) ? tangle->box.bottom_left_back.p[c] : tangle->box.top_right_front.p[c];
    rs.p[c] = 2 * w - r->p[c];
  }
  return rs;
}

void update_tangents_normals(struct tangle_state* tangle) {
  ov_clear_error();
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, false)) return;
  size_t n = (size_t)tangle->N;
  if (!ov_geometry(&s, s.pos.as<double>(), s.dxi.as<double>(), s.tan.as<double>(), s.nrm.as<double>()))
    return;
  if (download(&s, tangle->dxi, s.dxi, 8 * n) && download(&s, tangle->tangents, s.tan, 24 * n) &&
      download(&s, tangle->normals, s.nrm, 24 * n))
    sync(&s);
}

void update_tangent_normal(struct tangle_state* tangle, size_t k) {
  // The whole tangle's tangents are computed from the current positions and
  // node k's are written back (the reference computes node k from the stored
  // arc lengths; both agree whenever dxi is current).
  ov_clear_error();
  ov_state_impl& s = tls_state();
  if ((int)k < 0 || (int)k >= tangle->N) {
    ov_set_error(OV_ERR_INVALID, "update_tangent_normal: node %zu out of range", k);
    return;
  }
  if (tangle->status[k].status == EMPTY) return;
  if (!upload_tangle(&s, tangle, false)) return;
  if (!ov_geometry(&s, s.pos.as<double>(), s.dxi.as<double>(), s.tan.as<double>(), s.nrm.as<double>()))
    return;
  cudaMemcpyAsync(&tangle->tangents[k], s.tan.as<double>() + 3 * k, 24, cudaMemcpyDeviceToHost, s.stream);
  cudaMemcpyAsync(&tangle->normals[k], s.nrm.as<double>() + 3 * k, 24, cudaMemcpyDeviceToHost, s.stream);
  sync(&s);
}

void update_velocities(struct tangle_state* tangle, double t, struct octree* tree) {
  ov_clear_error();
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, true)) return;
  size_t n = (size_t)tangle->N;
  if (n == 0) return;
  if (!upload(&s, tangle->tangents, s.tan, 24 * n) || !upload(&s, tangle->normals, s.nrm, 24 * n)) return;
  OvTree* ext = (tree && s.P.use_bh) ? &tree->h.st.tree : nullptr;
  if (ext && tree->h.st.n != tangle->N) {
    ov_set_error(OV_ERR_INVALID, "octree built for %d slots, tangle has %d", tree->h.st.n, tangle->N);
    return;
  }
  if (!ov_velocities(&s, t, s.pos.as<double>(), s.dxi.as<double>(), s.tan.as<double>(),
                     s.nrm.as<double>(), s.vels.as<double>(), s.vs.as<double>(), ext))
    return;
  if (download(&s, tangle->vels, s.vels, 24 * n) && download(&s, tangle->vs, s.vs, 24 * n)) sync(&s);
}

void update_velocity(struct tangle_state* tangle, int k, double t, struct octree* tree) {
  // One node: its Biot-Savart sums as point queries at node k, then the same
  // epilogue restricted to slot k.  O(N (1 + images)) work, one call.
  ov_clear_error();
  if (!tangle || k < 0 || k >= tangle->N) {
    ov_set_error(OV_ERR_INVALID, "update_velocity: node %d out of range", k);
    return;
  }
  if (tangle->status[k].status == EMPTY) return;
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, true)) return;
  size_t n = (size_t)tangle->N;
  if (!upload(&s, tangle->tangents, s.tan, 24 * n) || !upload(&s, tangle->normals, s.nrm, 24 * n)) return;
  if (tree && s.P.use_bh && tree->h.st.n != tangle->N) {
    ov_set_error(OV_ERR_INVALID, "octree built for %d slots, tangle has %d", tree->h.st.n, tangle->N);
    return;
  }
  DevBuf skip;
  if (!skip.reserve(sizeof(int))) return;
  bool ok = ov_cuda_ok(cudaMemcpyAsync(skip.p, &k, sizeof(int), cudaMemcpyHostToDevice, s.stream),
                       "cudaMemcpyAsync");
  const double* pt = s.pos.as<double>() + 3 * (size_t)k;
  double* nl = s.v_nl.as<double>() + 3 * (size_t)k;
  double* im = s.v_img.as<double>() + 3 * (size_t)k;
  if (ok && !s.P.lia_only) {
    if (s.P.use_bh && tree)
      ok = ov_tree_walk_points(&s, &tree->h.st.tree, 1, pt, skip.as<int>(), s.P.theta, nl, im);
    else
      ok = ov_direct_points(&s, s.pos.as<double>(), 1, pt, skip.as<int>(), nullptr, 0, nl, im);
  }
  ok = ok && ov_epilogue(&s, t, s.pos.as<double>(), s.tan.as<double>(), s.nrm.as<double>(),
                         s.v_nl.as<double>(), s.v_img.as<double>(), s.vels.as<double>(),
                         s.vs.as<double>(), k, k + 1);
  if (ok) {
    cudaMemcpyAsync(&tangle->vels[k], s.vels.as<double>() + 3 * (size_t)k, 24, cudaMemcpyDeviceToHost,
                    s.stream);
    cudaMemcpyAsync(&tangle->vs[k], s.vs.as<double>() + 3 * (size_t)k, 24, cudaMemcpyDeviceToHost,
                    s.stream);
    sync(&s);
  }
  skip.release();
}

// calculate_vs_shift (src/tangle.c:553-576): the segments' velocity at
// r + shift, skipping node `skip`, over all nodes or the list
// use_only_points.  A point query on the device.
struct vec3d calculate_vs_shift(const struct tangle_state* tangle, struct vec3d r, int skip,
                                const struct vec3d* shift, const int* use_only_points,
                                const int Npoints) {
  ov_clear_error();
  struct vec3d out = {{0, 0, 0}};
  if (shift)
    for (int c = 0; c < 3; ++c) r.p[c] += shift->p[c];
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, false)) return out;
  DevBuf q;
  int npo = use_only_points ? Npoints : 0;
  for (int i = 0; i < npo; ++i) {
    if (use_only_points[i] < 0 || use_only_points[i] >= tangle->N) {
      ov_set_error(OV_ERR_INVALID, "calculate_vs_shift: node %d out of range", use_only_points[i]);
      return out;
    }
  }
  if (!q.reserve(sizeof(double) * 6 + sizeof(int) * (1 + (size_t)npo))) return out;
  double* dpt = q.as<double>();
  double* dout = dpt + 3;
  int* dskip = reinterpret_cast<int*>(dpt + 6);
  int* donly = dskip + 1;
  bool ok = ov_cuda_ok(cudaMemcpyAsync(dpt, r.p, 24, cudaMemcpyHostToDevice, s.stream), "copy") &&
            ov_cuda_ok(cudaMemcpyAsync(dskip, &skip, sizeof(int), cudaMemcpyHostToDevice, s.stream), "copy");
  if (ok && npo > 0)
    ok = ov_cuda_ok(cudaMemcpyAsync(donly, use_only_points, sizeof(int) * npo, cudaMemcpyHostToDevice,
                                    s.stream), "copy");
  ok = ok && ov_direct_points(&s, s.pos.as<double>(), 1, dpt, dskip, use_only_points ? donly : nullptr,
                              npo, dout, nullptr);
  ok = ok && ov_cuda_ok(cudaMemcpyAsync(out.p, dout, 24, cudaMemcpyDeviceToHost, s.stream), "copy") &&
       sync(&s);
  q.release();
  if (!ok) memset(&out, 0, sizeof(out));
  return out;
}

struct vec3d calculate_vs(struct tangle_state* tangle, struct vec3d r, int skip) {
  return calculate_vs_shift(tangle, r, skip, NULL, NULL, 0);
}

void euler_step(struct tangle_state* tangle, double dt) {
  ov_clear_error();
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, false)) return;
  size_t n = (size_t)tangle->N;
  if (n == 0) return;
  if (!upload(&s, tangle->vels, s.vels, 24 * n)) return;
  if (ov_euler(&s, dt) && download(&s, tangle->vnodes, s.pos, 24 * n)) sync(&s);
}

void rk4_step(struct tangle_state* tangle, double t, double dt) {
  ov_clear_error();
  ov_state_impl& s = tls_state();
  if (!upload_tangle(&s, tangle, true)) return;
  size_t n = (size_t)tangle->N;
  if (n == 0) return;
  if (!upload(&s, tangle->vels, s.vels, 24 * n)) return;
  if (ov_rk4(&s, t, dt, g_rk4_classic) && download(&s, tangle->vnodes, s.pos, 24 * n)) sync(&s);
}

struct octree* octree_build(const struct tangle_state* tangle, int quadtree) {
  ov_clear_error();
  octree* tr = new octree();
  ov_state_impl* s = &tr->h.st;
  int saved = global_BH_quadtree;
  global_BH_quadtree = quadtree;
  bool ok = upload_tangle(s, tangle, false);
  global_BH_quadtree = saved;
  ok = ok && ov_tree_build(s, s->pos.as<double>(), &s->tree) && sync(s);
  if (!ok) {
    state_release(s);
    delete tr;
    return nullptr;
  }
  return tr;
}

void octree_destroy(struct octree* tree) {
  if (!tree) return;
  state_release(&tree->h.st);
  delete tree;
}

void octree_get_vs(const struct octree* tree, const struct vec3d* r, double resolution,
                   struct vec3d* res, int skip) {
  ov_clear_error();
  if (!res) return;
  memset(res, 0, sizeof(*res));
  if (!tree || !r) return;
  ov_state_impl* s = const_cast<ov_state_impl*>(&tree->h.st);
  s->P.precision = g_precision;
  DevBuf q;
  if (!q.reserve(sizeof(double) * 6 + sizeof(int))) return;
  double* dpt = q.as<double>();
  int* dskip = reinterpret_cast<int*>(dpt + 6);
  bool ok = ov_cuda_ok(cudaMemcpyAsync(dpt, r->p, 24, cudaMemcpyHostToDevice, s->stream), "copy") &&
            ov_cuda_ok(cudaMemcpyAsync(dskip, &skip, sizeof(int), cudaMemcpyHostToDevice, s->stream), "copy");
  ok = ok && ov_tree_walk_points(s, &s->tree, 1, dpt, dskip, resolution, dpt + 3, nullptr);
  ok = ok && ov_cuda_ok(cudaMemcpyAsync(res->p, dpt + 3, 24, cudaMemcpyDeviceToHost, s->stream), "copy") &&
       sync(s);
  q.release();
  if (!ok) memset(res, 0, sizeof(*res));
}

}  // extern "C"
