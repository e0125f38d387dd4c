// C-ABI entry points (include/buffem_b200.h).  Argument checking, ownership
// and error reporting live here; all compute is dispatched to the CUDA
// kernels.  No exception crosses the ABI; errors are status codes plus a
// thread-local message.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <strings.h>
#include <vector>

#include "internal.h"

namespace bg {

static thread_local std::string t_err;
std::atomic<long long> g_launches{0};

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
}

static cudaStream_t s_stream = nullptr;
static std::mutex s_mu;
static int s_dev_ok = 0;

int ensure_device() {
  std::lock_guard<std::mutex> lk(s_mu);
  if (s_dev_ok) return BG_OK;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error("no CUDA device available (%s); this library has no CPU fallback",
              e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
    return BG_ERR_CUDA;
  }
  int dev = 0;
  BG_CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceProp p;
  BG_CUDA_TRY(cudaGetDeviceProperties(&p, dev));
  if (p.major < 10) {
    set_error("device %s (sm_%d%d) is not sm_100a; kernels are built for B200 only", p.name, p.major, p.minor);
    return BG_ERR_CUDA;
  }
  BG_CUDA_TRY(cudaStreamCreateWithFlags(&s_stream, cudaStreamNonBlocking));
  // keep up to 8 GiB of freed stream-ordered allocations in this process's
  // default pool across synchronizations, so per-call scratch buffers do not
  // go back to the driver every call (larger transients are still returned)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = 8ull << 30;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  s_dev_ok = 1;
  return BG_OK;
}

// A calling thread may direct the library's work to another stream (the
// batched sweeps run several slots concurrently); by default everything runs
// on the library stream.
static thread_local cudaStream_t t_stream = nullptr;
cudaStream_t stream() { return t_stream ? t_stream : s_stream; }
void set_thread_stream(cudaStream_t s) { t_stream = s; }

// ------------------------------------------------------------- profiling
struct ProfRec { cudaEvent_t a, b; int cls; double flops; };
static bool s_prof = false;
static std::vector<ProfRec> s_recs;
static std::vector<cudaEvent_t> s_pool;
static cudaEvent_t s_open[PROF_NCLASS];
static cudaEvent_t take_event() {
  if (!s_pool.empty()) { cudaEvent_t e = s_pool.back(); s_pool.pop_back(); return e; }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
bool prof_on() { return s_prof; }
void prof_start(int cls) {
  if (!s_prof) return;
  s_open[cls] = take_event();
  cudaEventRecord(s_open[cls], stream());
}
void prof_stop(int cls, double flops) {
  if (!s_prof) return;
  cudaEvent_t e = take_event();
  cudaEventRecord(e, stream());
  s_recs.push_back(ProfRec{s_open[cls], e, cls, flops});
}

}  // namespace bg

using namespace bg;

extern "C" {

const char *bg_last_error(void) { return t_err.c_str(); }

static int finish_geometry(bg_geometry *g) {
  g->bfOffset.assign(g->objs.size() + 1, 0);
  g->vOffset.assign(g->objs.size() + 1, 0);
  g->tOffset.assign(g->objs.size() + 1, 0);
  for (size_t i = 0; i < g->objs.size(); i++) {
    g->bfOffset[i + 1] = g->bfOffset[i] + g->objs[i].nif;
    g->vOffset[i + 1] = g->vOffset[i] + g->objs[i].nv;
    g->tOffset[i + 1] = g->tOffset[i] + g->objs[i].nt;
  }
  g->N = g->bfOffset.back();
  g->NV = g->vOffset.back();
  g->NT = g->tOffset.back();
  if (g->N <= 0) { set_error("geometry has no interior faces"); return BG_ERR_ARG; }
  return BG_OK;
}

static int check_material(const bg_material &m) {
  if (m.kind < BG_MAT_CONST_ISO || m.kind > BG_MAT_GAUSSIAN) { set_error("unknown material kind %d", m.kind); return BG_ERR_ARG; }
  if (m.kind == BG_MAT_GAUSSIAN && !(m.width > 0)) { set_error("gaussian material needs width > 0"); return BG_ERR_ARG; }
  return BG_OK;
}

// xf: 12 doubles per object (one-time transformation, M row-major then D) or
// null; labels: one per object or null (the mesh file name is the label then,
// as SWGVolume's constructor does without one)
static int create_objects(int nobj, const char *const *meshfiles, const double *xf, const bg_material *materials,
                          const std::string *labels, const std::shared_ptr<const MatPropFn> *matprops,
                          const std::shared_ptr<const SVTensorFn> *svts, bg_geometry **out) {
  *out = nullptr;
  bg_geometry *g = new (std::nothrow) bg_geometry();
  if (!g) { set_error("out of host memory"); return BG_ERR_NOMEM; }
  g->objs.resize(nobj);
  for (int i = 0; i < nobj; i++) {
    if (!meshfiles[i]) { delete g; set_error("mesh file %d is NULL", i); return BG_ERR_ARG; }
    // BG_MAT_EXPR comes only with a position-dependent SVTENSOR file
    int st = (svts && svts[i] && materials[i].kind == BG_MAT_EXPR) ? BG_OK : check_material(materials[i]);
    if (!st) st = load_object(g->objs[i], meshfiles[i], xf ? xf + 12 * i : nullptr);
    if (st) { delete g; return st; }
    g->objs[i].mat = materials[i];
    g->objs[i].label = labels ? labels[i] : std::string(meshfiles[i]);
    if (matprops && matprops[i]) {
      g->objs[i].matprop = matprops[i];
      g->dispersive = true;
    }
    if (svts && svts[i]) {
      g->objs[i].svt = svts[i];
      g->dispersive = true;
    }
  }
  int st = finish_geometry(g);
  if (st) { delete g; return st; }
  *out = g;
  return BG_OK;
}

int bg_geometry_create_objects(int nobj, const char *const *meshfiles, const double *displacements,
                               const bg_material *materials, bg_geometry **out) {
  if (!out || nobj <= 0 || !meshfiles || !materials) { set_error("bg_geometry_create_objects: bad arguments"); return BG_ERR_ARG; }
  if (!displacements) return create_objects(nobj, meshfiles, nullptr, materials, nullptr, nullptr, nullptr, out);
  std::vector<double> xf(12 * (size_t)nobj, 0.0);
  for (int i = 0; i < nobj; i++) {
    double *x = &xf[12 * (size_t)i];
    x[0] = x[4] = x[8] = 1.0;
    for (int k = 0; k < 3; k++) x[9 + k] = displacements[3 * i + k];
  }
  return create_objects(nobj, meshfiles, xf.data(), materials, nullptr, nullptr, nullptr, out);
}

static int create_from_objects(std::vector<GeoObject> &objs, bg_geometry **out);

int bg_geometry_create(const char *path, bg_geometry **out) {
  if (!path || !out) { set_error("bg_geometry_create: bad arguments"); return BG_ERR_ARG; }
  *out = nullptr;
  std::vector<GeoObject> objs;
  int st = parse_buffgeo(path, objs);
  if (st) return st;
  return create_from_objects(objs, out);
}

int bg_trans_file_count(const char *trans_path) {
  if (!trans_path) { set_error("bg_trans_file_count: bad arguments"); return BG_ERR_ARG; }
  std::vector<TransEntry> tr;
  int st = parse_trans_file(trans_path, tr);
  return st ? st : (int)tr.size();
}

int bg_trans_file_tag(const char *trans_path, int k, char *buf, int cap) {
  if (!trans_path || k < 0 || cap < 0 || (cap > 0 && !buf)) { set_error("bg_trans_file_tag: bad arguments"); return BG_ERR_ARG; }
  std::vector<TransEntry> tr;
  int st = parse_trans_file(trans_path, tr);
  if (st) return st;
  if (k >= (int)tr.size()) { set_error("bg_trans_file_tag: %s has %d transformations", trans_path, (int)tr.size()); return BG_ERR_ARG; }
  const std::string &t = tr[k].tag;
  if (cap > 0) {
    size_t n = std::min(t.size(), (size_t)cap - 1);
    std::memcpy(buf, t.data(), n);
    buf[n] = 0;
  }
  return (int)t.size();
}

int bg_geometry_create_transformed(const char *path, const char *trans_path, int k, bg_geometry **out) {
  if (!path || !trans_path || !out || k < 0) { set_error("bg_geometry_create_transformed: bad arguments"); return BG_ERR_ARG; }
  *out = nullptr;
  std::vector<GeoObject> objs;
  int st = parse_buffgeo(path, objs);
  if (st) return st;
  std::vector<TransEntry> tr;
  if ((st = parse_trans_file(trans_path, tr))) return st;
  if (k >= (int)tr.size()) {
    set_error("bg_geometry_create_transformed: %s has %d transformations", trans_path, (int)tr.size());
    return BG_ERR_ARG;
  }
  if ((st = apply_trans(tr[k], objs))) return st;
  return create_from_objects(objs, out);
}

static int create_from_objects(std::vector<GeoObject> &objs, bg_geometry **out) {
  std::vector<const char *> names;
  std::vector<double> xf;
  std::vector<bg_material> mats;
  std::vector<std::string> labels;
  std::vector<std::shared_ptr<const MatPropFn>> matprops;
  std::vector<std::shared_ptr<const SVTensorFn>> svts;
  for (auto &o : objs) {
    names.push_back(o.mesh.c_str());
    xf.insert(xf.end(), o.xf, o.xf + 12);
    mats.push_back(o.mat);
    labels.push_back(o.label);
    matprops.push_back(o.matprop);
    svts.push_back(o.svt);
  }
  return create_objects((int)objs.size(), names.data(), xf.data(), mats.data(), labels.data(), matprops.data(),
                        svts.data(), out);
}

static void dfree(void *p) { if (p) cudaFree(p); }

void bg_geometry_destroy(bg_geometry *g) {
  if (!g) return;
  DevGeom &d = g->dev;
  dfree(d.V4); dfree(d.tetVI); dfree(d.tetVol); dfree(d.tetP4); dfree(d.tetObj); dfree(d.bfTet);
  dfree(d.bfQ); dfree(d.bfLoc); dfree(d.tetFI); dfree(d.bfV); dfree(d.bfArea); dfree(d.bfRadius); dfree(d.mats); dfree(d.expr); dfree(d.objOrigin);
  dfree(d.tileTet); dfree(d.tileNT); dfree(d.bfTileLoc);
  NearData &n = g->near;
  dfree(n.pairs); dfree(n.pairTP); dfree(n.fibbi); dfree(n.tp); dfree(n.tpOrdA); dfree(n.tpOrdB); dfree(n.tpMom); dfree(n.tpFlag);
  dfree(g->graph.rowptr); dfree(g->graph.col); dfree(g->graph.etr);
  dfree(g->d_scratch);
  dfree(g->d_fieldTet); dfree(g->d_fieldFace);
  gnn_cache_free(g);
  delete g;
}

int bg_geometry_num_bfs(const bg_geometry *g) { return g ? g->N : BG_ERR_ARG; }
int bg_geometry_num_objects(const bg_geometry *g) { return g ? (int)g->objs.size() : BG_ERR_ARG; }
int bg_geometry_bf_offset(const bg_geometry *g, int obj) {
  if (!g || obj < 0 || obj > (int)g->objs.size()) { set_error("bad object index"); return BG_ERR_ARG; }
  return g->bfOffset[obj];
}

int bg_geometry_material_eps(const bg_geometry *g, int obj, double omega_re, double omega_im, double *eps) {
  if (!g || !eps || obj < 0 || obj >= (int)g->objs.size()) {
    set_error("bg_geometry_material_eps: bad arguments");
    return BG_ERR_ARG;
  }
  const Object &o = g->objs[obj];
  if (o.matprop) { matprop_eps(*o.matprop, omega_re, omega_im, eps); return 1; }
  if (o.svt) {
    // the scalar SVTensor::Evaluate(Omega, x) returns the xx component
    // (SVTensor.cc:375-380); this query has no point, so a position-dependent
    // tensor is taken at the origin of coordinates (bg_geometry_material_tensor
    // takes one)
    double Q[18];
    const double x0[3] = {0.0, 0.0, 0.0};
    svtensor_eval(*o.svt, omega_re, omega_im, x0, Q);
    eps[0] = Q[0];
    eps[1] = Q[1];
    return 1;
  }
  if (o.mat.kind == BG_MAT_CONST_ISO) { eps[0] = o.mat.eps[0]; eps[1] = o.mat.eps[1]; return 0; }
  set_error("bg_geometry_material_eps: object %d has a tensor or position-dependent permittivity", obj);
  return BG_ERR_ARG;
}

int bg_geometry_material_tensor(const bg_geometry *g, int obj, double omega_re, double omega_im, const double *x,
                                double *Q) {
  if (!g || !x || !Q || obj < 0 || obj >= (int)g->objs.size()) {
    set_error("bg_geometry_material_tensor: bad arguments");
    return BG_ERR_ARG;
  }
  const Object &o = g->objs[obj];
  for (int k = 0; k < 18; k++) Q[k] = 0.0;
  if (o.svt) { svtensor_eval(*o.svt, omega_re, omega_im, x, Q); return BG_OK; }
  double e[2];
  const bg_material &m = o.mat;
  if (o.matprop) {
    matprop_eps(*o.matprop, omega_re, omega_im, e);
  } else if (m.kind == BG_MAT_CONST_TENSOR) {
    // as the device evaluates it: off-diagonal pairs averaged
    for (int k = 0; k < 18; k++) Q[k] = m.eps[k];
    for (int a = 0; a < 3; a++) {
      int b = (a + 1) % 3;
      for (int c = 0; c < 2; c++) {
        double avg = 0.5 * (Q[2 * (3 * a + b) + c] + Q[2 * (3 * b + a) + c]);
        Q[2 * (3 * a + b) + c] = Q[2 * (3 * b + a) + c] = avg;
      }
    }
    return BG_OK;
  } else if (m.kind == BG_MAT_JANUS_Z) {
    bool up = x[2] > m.center[2];
    e[0] = up ? m.eps[0] : m.eps2[0];
    e[1] = up ? m.eps[1] : m.eps2[1];
  } else if (m.kind == BG_MAT_GAUSSIAN) {
    double d0 = x[0] - m.center[0], d1 = x[1] - m.center[1], d2 = x[2] - m.center[2];
    double gs = std::exp(-(d0 * d0 + d1 * d1 + d2 * d2) / (m.width * m.width));
    e[0] = m.eps[0] + m.amp[0] * gs;
    e[1] = m.eps[1] + m.amp[1] * gs;
  } else {
    e[0] = m.eps[0];
    e[1] = m.eps[1];
  }
  for (int a = 0; a < 3; a++) { Q[2 * (4 * a)] = e[0]; Q[2 * (4 * a) + 1] = e[1]; }
  return BG_OK;
}

int bg_geometry_object_index(const bg_geometry *g, const char *label) {
  if (!g || !label) { set_error("bg_geometry_object_index: bad arguments"); return BG_ERR_ARG; }
  for (size_t i = 0; i < g->objs.size(); i++)
    if (!strcasecmp(label, g->objs[i].label.c_str())) return (int)i;
  set_error("no object labelled %s", label);
  return BG_ERR_ARG;
}

int bg_geometry_object_label(const bg_geometry *g, int obj, char *buf, int cap) {
  if (!g || obj < 0 || obj >= (int)g->objs.size() || cap < 0 || (cap > 0 && !buf)) {
    set_error("bg_geometry_object_label: bad arguments");
    return BG_ERR_ARG;
  }
  const std::string &l = g->objs[obj].label;
  if (cap > 0) {
    size_t n = std::min(l.size(), (size_t)cap - 1);
    std::memcpy(buf, l.data(), n);
    buf[n] = 0;
  }
  return (int)l.size();
}

int bg_geometry_vertices(const bg_geometry *g, int obj, double *xyz, double *origin) {
  if (!g || obj < 0 || obj >= (int)g->objs.size()) { set_error("bg_geometry_vertices: bad arguments"); return BG_ERR_ARG; }
  const Object &o = g->objs[obj];
  if (xyz) std::memcpy(xyz, o.V.data(), sizeof(double) * o.V.size());
  if (origin) for (int k = 0; k < 3; k++) origin[k] = o.origin[k];
  return o.nv;
}

int bg_geometry_faces(const bg_geometry *g, int obj, int *out) {
  if (!g || !out || obj < 0 || obj >= (int)g->objs.size()) { set_error("bg_geometry_faces: bad arguments"); return BG_ERR_ARG; }
  const Object &o = g->objs[obj];
  for (int i = 0; i < o.nif; i++) {
    const Face &F = o.F[i];
    int *q = out + 9 * i;
    q[0] = F.iV1; q[1] = F.iV2; q[2] = F.iV3; q[3] = F.iQP; q[4] = F.iQM;
    q[5] = F.iPTet; q[6] = F.iMTet; q[7] = F.PIndex; q[8] = F.MIndex;
  }
  return BG_OK;
}

int bg_geometry_set_singular_order(bg_geometry *g, int n) {
  if (!g || n < 2 || n > 16) { set_error("singular order must be in [2,16]"); return BG_ERR_ARG; }
  if (g->sing_refine && n > 14) { set_error("with the refined singular rule the order must be in [2,14] (orders n and n+2 are used)"); return BG_ERR_ARG; }
  if (g->precomputed && n != g->singular_order) { set_error("singular order must be set before the precompute"); return BG_ERR_STATE; }
  g->singular_order = n;
  return BG_OK;
}

int bg_geometry_set_singular_refine(bg_geometry *g, int on, double flag_tol, double tol) {
  if (!g || (on != 0 && on != 1)) { set_error("bg_geometry_set_singular_refine: bad arguments"); return BG_ERR_ARG; }
  if (on && !(flag_tol > 0.0 && tol > 0.0 && flag_tol < 1.0 && tol < 1.0)) {
    set_error("bg_geometry_set_singular_refine: tolerances must be in (0, 1)");
    return BG_ERR_ARG;
  }
  if (on && g->singular_order > 14) { set_error("with the refined singular rule the order must be in [2,14] (orders n and n+2 are used)"); return BG_ERR_ARG; }
  bool same = (bool)on == g->sing_refine && (!on || (flag_tol == g->sing_flag_tol && tol == g->sing_tol));
  if (g->precomputed && !same) { set_error("the singular rule must be set before the precompute"); return BG_ERR_STATE; }
  g->sing_refine = on != 0;
  if (on) { g->sing_flag_tol = flag_tol; g->sing_tol = tol; }
  return BG_OK;
}

int bg_geometry_singular_stats(bg_geometry *g, long long *out) {
  if (!g || !out) { set_error("bg_geometry_singular_stats: bad arguments"); return BG_ERR_ARG; }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  for (int i = 0; i < 6; i++) out[i] = g->sing_stats[i];
  return BG_OK;
}

int bg_geometry_singular_moments(bg_geometry *g, int *count, int *pairs, int *verts, double *mom) {
  if (!g || !count) { set_error("bg_geometry_singular_moments: bad arguments"); return BG_ERR_ARG; }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  const NearData &nd = g->near;
  int ns = nd.ntp - nd.ntp_reg;
  *count = ns;
  if (ns <= 0) return BG_OK;
  if (pairs) {
    std::vector<int4> tp(ns);
    std::vector<unsigned char> fl(ns);
    BG_CUDA_TRY(cudaMemcpy(tp.data(), nd.tp + nd.ntp_reg, sizeof(int4) * ns, cudaMemcpyDeviceToHost));
    BG_CUDA_TRY(cudaMemcpy(fl.data(), nd.tpFlag, (size_t)ns, cudaMemcpyDeviceToHost));
    for (int i = 0; i < ns; i++) {
      pairs[4 * i] = tp[i].x; pairs[4 * i + 1] = tp[i].y; pairs[4 * i + 2] = tp[i].z; pairs[4 * i + 3] = fl[i];
    }
  }
  if (verts) {
    std::vector<int4> a(ns), b(ns);
    BG_CUDA_TRY(cudaMemcpy(a.data(), nd.tpOrdA + nd.ntp_reg, sizeof(int4) * ns, cudaMemcpyDeviceToHost));
    BG_CUDA_TRY(cudaMemcpy(b.data(), nd.tpOrdB + nd.ntp_reg, sizeof(int4) * ns, cudaMemcpyDeviceToHost));
    for (int i = 0; i < ns; i++) {
      int *q = verts + 8 * i;
      q[0] = a[i].x; q[1] = a[i].y; q[2] = a[i].z; q[3] = a[i].w;
      q[4] = b[i].x; q[5] = b[i].y; q[6] = b[i].z; q[7] = b[i].w;
    }
  }
  if (mom) BG_CUDA_TRY(cudaMemcpy(mom, nd.tpMom + 24 * (size_t)nd.ntp_reg, sizeof(double) * 24 * ns, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_geometry_precompute(bg_geometry *g) {
  if (!g) { set_error("null geometry"); return BG_ERR_ARG; }
  if (g->precomputed) return BG_OK;
  int st = upload_geometry(g);
  if (!st) st = build_near_lists(g);
  if (!st) st = precompute_near(g);
  if (!st) g->precomputed = true;
  return st;
}

int bg_geometry_near_data(bg_geometry *g, int *count, int *pairs, double *data) {
  if (!g || !count) { set_error("bg_geometry_near_data: bad arguments"); return BG_ERR_ARG; }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  *count = g->near.npairs;
  if (pairs) BG_CUDA_TRY(cudaMemcpy(pairs, g->near.pairs, sizeof(int2) * g->near.npairs, cudaMemcpyDeviceToHost));
  if (data) BG_CUDA_TRY(cudaMemcpy(data, g->near.fibbi, sizeof(double) * 6 * g->near.npairs, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_matrix_create(bg_geometry *g, int precision, bg_matrix **out) {
  if (!g || !out || (precision != BG_C128 && precision != BG_C64)) { set_error("bg_matrix_create: bad arguments"); return BG_ERR_ARG; }
  *out = nullptr;
  int st = ensure_device();
  if (st) return st;
  bg_matrix *m = new (std::nothrow) bg_matrix();
  if (!m) { set_error("out of host memory"); return BG_ERR_NOMEM; }
  m->g = g;
  m->N = g->N;
  m->precision = precision;
  // complex64 storage feeds TMA: 16-byte aligned column starts need an even,
  // here 32-aligned, leading dimension
  m->ld = precision == BG_C128 ? (size_t)g->N : ((size_t)g->N + 31) / 32 * 32;
  size_t esz = precision == BG_C128 ? 16 : 8;
  cudaError_t e = cudaMalloc(&m->d, esz * m->ld * (size_t)m->N);
  if (e != cudaSuccess) {
    delete m;
    set_error("cannot allocate %.2f GB matrix on the device: %s", esz * (double)g->N * g->N / 1e9, cudaGetErrorString(e));
    return BG_ERR_NOMEM;
  }
  if (m->ld > (size_t)m->N) {
    // the padding rows N .. ld-1 are zero for good: no kernel writes them, and
    // the symmetric complex64 product copies one of them with an odd N
    e = cudaMemset2DAsync((char *)m->d + esz * (size_t)m->N, esz * m->ld, 0, esz * (m->ld - (size_t)m->N), m->N,
                          stream());
    if (e != cudaSuccess) { cudaFree(m->d); delete m; set_error("cudaMemset2DAsync: %s", cudaGetErrorString(e)); return BG_ERR_CUDA; }
  }
  e = cudaMalloc(&m->d_ipiv, sizeof(int) * (size_t)m->N);
  if (e != cudaSuccess) { cudaFree(m->d); delete m; set_error("cannot allocate pivots"); return BG_ERR_NOMEM; }
  *out = m;
  return BG_OK;
}

void bg_matrix_destroy(bg_matrix *m) {
  if (!m) return;
  dfree(m->d); dfree(m->d_ipiv); dfree(m->d_work); dfree(m->d_perm);
  delete m;
}

int bg_assemble(bg_geometry *g, double wr, double wi, bg_matrix *m) {
  if (!g || !m) { set_error("bg_assemble: null argument"); return BG_ERR_ARG; }
  if (m->g != g && m->N != g->N) { set_error("wrong-size matrix passed to bg_assemble (%d != %d)", m->N, g->N); return BG_ERR_ARG; }
  if (m->N != g->N) { set_error("wrong-size matrix passed to bg_assemble (%d != %d)", m->N, g->N); return BG_ERR_ARG; }
  if (m->precision != BG_C128) { set_error("bg_assemble: only complex128 matrices are assembled here"); return BG_ERR_ARG; }
  if (wr == 0.0 && wi == 0.0) { set_error("bg_assemble: omega must be nonzero"); return BG_ERR_ARG; }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  m->factored = false;
  prof_start(PROF_ASM_FAR);
  st = assemble_far(g, wr, wi, m->d, m->ld);
  prof_stop(PROF_ASM_FAR, 64.0 * g->N * (double)g->N);
  prof_start(PROF_ASM_NEAR);
  if (!st) st = assemble_near(g, wr, wi, m->d, m->ld);
  if (!st) st = assemble_gram(g, wr, wi, m->d, m->ld);
  prof_stop(PROF_ASM_NEAR, 0.0);
  m->symmetric = !st;   // far, near and Gram entries are written symmetrically
  return st;
}

int bg_assemble_with_copy(bg_geometry *g, double wr, double wi, bg_matrix *m, bg_matrix *f) {
  if (!g || !m || !f) { set_error("bg_assemble_with_copy: null argument"); return BG_ERR_ARG; }
  if (m->N != g->N || f->N != g->N) {
    set_error("wrong-size matrix passed to bg_assemble_with_copy (%d, %d != %d)", m->N, f->N, g->N);
    return BG_ERR_ARG;
  }
  if (m->precision != BG_C128 || f->precision != BG_C64) {
    set_error("bg_assemble_with_copy: a complex128 matrix and a complex64 copy are required");
    return BG_ERR_ARG;
  }
  if (wr == 0.0 && wi == 0.0) { set_error("bg_assemble_with_copy: omega must be nonzero"); return BG_ERR_ARG; }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  m->factored = false;
  f->factored = false;
  prof_start(PROF_ASM_FAR);
  st = assemble_far(g, wr, wi, m->d, m->ld, nullptr, f->d, f->ld);
  prof_stop(PROF_ASM_FAR, 64.0 * g->N * (double)g->N);
  prof_start(PROF_ASM_NEAR);
  if (!st) st = assemble_near(g, wr, wi, m->d, m->ld, nullptr, f->d, f->ld);
  if (!st) st = assemble_gram(g, wr, wi, m->d, m->ld, nullptr, f->d, f->ld);
  prof_stop(PROF_ASM_NEAR, 0.0);
  m->symmetric = !st;
  f->symmetric = !st;
  return st;
}

int bg_matrix_download(const bg_matrix *m, void *host) {
  if (!m || !host) { set_error("bg_matrix_download: bad arguments"); return BG_ERR_ARG; }
  size_t esz = m->precision == BG_C128 ? 16 : 8;
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy2D(host, esz * m->N, m->d, esz * m->ld, esz * m->N, m->N, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_matrix_get_rows(const bg_matrix *m, int nrows, const int *rows, void *host) {
  if (!m || nrows < 0 || (nrows > 0 && (!rows || !host))) { set_error("bg_matrix_get_rows: bad arguments"); return BG_ERR_ARG; }
  for (int k = 0; k < nrows; k++)
    if (rows[k] < 0 || rows[k] >= m->N) { set_error("bg_matrix_get_rows: row %d out of range", rows[k]); return BG_ERR_ARG; }
  size_t esz = m->precision == BG_C128 ? 16 : 8;
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  // row r of the column-major matrix: N elements esz bytes wide, ld elements apart
  for (int k = 0; k < nrows; k++)
    BG_CUDA_TRY(cudaMemcpy2D((char *)host + esz * (size_t)m->N * k, esz, (const char *)m->d + esz * (size_t)rows[k],
                             esz * m->ld, esz, m->N, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_matrix_upload(bg_matrix *m, const void *host) {
  if (!m || !host) { set_error("bg_matrix_upload: bad arguments"); return BG_ERR_ARG; }
  size_t esz = m->precision == BG_C128 ? 16 : 8;
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy2D(m->d, esz * m->ld, host, esz * m->N, esz * m->N, m->N, cudaMemcpyHostToDevice));
  m->factored = false;
  m->symmetric = false;
  return BG_OK;
}

int bg_matrix_convert(const bg_matrix *src, bg_matrix *dst) {
  if (!src || !dst) { set_error("bg_matrix_convert: null matrix"); return BG_ERR_ARG; }
  return matrix_convert(src, dst);
}

int bg_lu_solve_refined_device(bg_matrix *A, bg_matrix *F, void *dB, int ldb, int nrhs, double tol, int maxit,
                               double *stats) {
  if (!A || !F || !dB || nrhs <= 0 || ldb < A->N || maxit < 1) { set_error("bg_lu_solve_refined: bad arguments"); return BG_ERR_ARG; }
  if (A->precision != BG_C128 || F->precision != BG_C64 || A->N != F->N) {
    set_error("bg_lu_solve_refined: needs a complex128 matrix and complex64 factors of the same size");
    return BG_ERR_ARG;
  }
  if (!F->factored) { set_error("bg_lu_solve_refined: factors missing (call bg_lu_factor on the complex64 matrix)"); return BG_ERR_STATE; }
  if (F->info > 0) { set_error("bg_lu_solve_refined: singular factors (info=%d)", F->info); return BG_ERR_NUMERIC; }
  return solve_refined(A, F, dB, ldb, nrhs, tol, maxit, stats);
}

int bg_lu_solve_refined(bg_matrix *A, bg_matrix *F, double *B, int nrhs, double tol, int maxit, double *stats) {
  if (!A || !B || nrhs <= 0) { set_error("bg_lu_solve_refined: bad arguments"); return BG_ERR_ARG; }
  size_t bytes = 16 * (size_t)A->N * nrhs;
  void *dB = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&dB, bytes, stream()));
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = bg_lu_solve_refined_device(A, F, dB, A->N, nrhs, tol, maxit, stats);
  if (!st) {
    e = cudaMemcpyAsync(B, dB, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(dB, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("refined solve: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_matrix_device_ptr(bg_matrix *m, void **dptr, int *ld) {
  if (!m || !dptr || !ld) { set_error("bg_matrix_device_ptr: bad arguments"); return BG_ERR_ARG; }
  *dptr = m->d;
  *ld = (int)m->ld;
  m->symmetric = false;   // the caller may write through the pointer
  return BG_OK;
}

int bg_lu_factor(bg_matrix *m) {
  if (!m) { set_error("bg_lu_factor: null matrix"); return BG_ERR_ARG; }
  m->symmetric = false;
  int st = lu_factor(m);
  if (st < 0) return st;
  m->factored = true;
  m->info = st;
  return st;
}

int bg_lu_pivots(const bg_matrix *m, int *ipiv) {
  if (!m || !ipiv) { set_error("bg_lu_pivots: bad arguments"); return BG_ERR_ARG; }
  if (!m->factored) { set_error("matrix is not factored"); return BG_ERR_STATE; }
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  BG_CUDA_TRY(cudaMemcpy(ipiv, m->d_ipiv, sizeof(int) * m->N, cudaMemcpyDeviceToHost));
  return BG_OK;
}

int bg_lu_solve_device(bg_matrix *m, void *dB, int ldb, int nrhs) {
  if (!m || !dB || nrhs <= 0 || ldb < m->N) { set_error("bg_lu_solve_device: bad arguments"); return BG_ERR_ARG; }
  if (!m->factored) { set_error("bg_lu_solve: matrix is not LU-factored"); return BG_ERR_STATE; }
  if (m->info > 0) { set_error("bg_lu_solve: factorization is singular (info=%d)", m->info); return BG_ERR_NUMERIC; }
  int st = lu_solve(m, dB, ldb, nrhs);
  if (!st) st = lu_solve_status(m);
  return st;
}

int bg_lu_solve_device_noalloc(bg_matrix *m, void *dB, int ldb, int nrhs) {
  if (!m || !dB || nrhs <= 0 || ldb < m->N) { set_error("bg_lu_solve_device_noalloc: bad arguments"); return BG_ERR_ARG; }
  int st = lu_noalloc_check(m, nrhs);
  if (st) return st;
  if (!m->factored) { set_error("bg_lu_solve_device_noalloc: matrix is not LU-factored"); return BG_ERR_STATE; }
  if (m->info > 0) { set_error("bg_lu_solve_device_noalloc: factorization is singular (info=%d)", m->info); return BG_ERR_NUMERIC; }
  return lu_solve_noalloc(m, dB, ldb, nrhs);
}

int bg_precond_create_jacobi(bg_matrix *A, bg_precond **out) {
  if (!A || !out || A->precision != BG_C128) { set_error("bg_precond_create_jacobi: complex128 matrix required"); return BG_ERR_ARG; }
  *out = nullptr;
  return precond_jacobi(A, out);
}

void bg_precond_destroy(bg_precond *P) {
  if (!P) return;
  // the arrays are stream-ordered allocations: freed after the work queued on
  // the library stream, without a device-wide synchronisation
  if (ensure_device() == BG_OK) {
    if (P->rowptr) cudaFreeAsync(P->rowptr, stream());
    if (P->col) cudaFreeAsync(P->col, stream());
    if (P->val) cudaFreeAsync(P->val, stream());
  }
  delete P;
}

int bg_precond_nnz(const bg_precond *P) { return P ? P->nnz : BG_ERR_ARG; }

int bg_gmres_solve_device(bg_matrix *A, const bg_precond *P, void *dB, int ldb, int nrhs, double tol, int restart,
                          int maxit, double *stats) {
  if (!A || !dB || nrhs <= 0 || ldb < A->N || restart < 2 || maxit < 1 || !(tol > 0)) {
    set_error("bg_gmres_solve: bad arguments");
    return BG_ERR_ARG;
  }
  if (A->precision != BG_C128) { set_error("bg_gmres_solve: complex128 matrix required"); return BG_ERR_ARG; }
  if (A->factored) { set_error("bg_gmres_solve: the matrix holds LU factors, not the operator"); return BG_ERR_STATE; }
  if (P && P->N != A->N) { set_error("bg_gmres_solve: preconditioner size mismatch"); return BG_ERR_ARG; }
  return gmres_solve(A, P, dB, ldb, nrhs, tol, restart, maxit, stats);
}

int bg_gmres_solve(bg_matrix *A, const bg_precond *P, double *B, int nrhs, double tol, int restart, int maxit,
                   double *stats) {
  if (!A || !B || nrhs <= 0) { set_error("bg_gmres_solve: bad arguments"); return BG_ERR_ARG; }
  size_t bytes = 16 * (size_t)A->N * nrhs;
  void *dB = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&dB, bytes, stream()));
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = bg_gmres_solve_device(A, P, dB, A->N, nrhs, tol, restart, maxit, stats);
  if (!st) {
    e = cudaMemcpyAsync(B, dB, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(dB, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_gmres_solve_mixed_device(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *dB, int ldb, int nrhs,
                                double tol, int restart, int maxit, double inner_tol, double *stats) {
  if (!A || !F || !dB || nrhs <= 0 || ldb < A->N || restart < 2 || maxit < 1 || !(tol > 0) || !(inner_tol > 0) ||
      !(inner_tol < 1)) {
    set_error("bg_gmres_solve_mixed: bad arguments");
    return BG_ERR_ARG;
  }
  if (A->precision != BG_C128 || F->precision != BG_C64 || F->N != A->N) {
    set_error("bg_gmres_solve_mixed: complex128 A and complex64 F of equal size required");
    return BG_ERR_ARG;
  }
  if (A->factored || F->factored) {
    set_error("bg_gmres_solve_mixed: the matrices hold LU factors, not the operator");
    return BG_ERR_STATE;
  }
  if (P && P->N != A->N) { set_error("bg_gmres_solve_mixed: preconditioner size mismatch"); return BG_ERR_ARG; }
  return gmres_solve_mixed(A, F, P, dB, ldb, nrhs, tol, restart, maxit, inner_tol, stats);
}

int bg_gmres_solve_mixed(bg_matrix *A, bg_matrix *F, const bg_precond *P, double *B, int nrhs, double tol,
                         int restart, int maxit, double inner_tol, double *stats) {
  if (!A || !B || nrhs <= 0) { set_error("bg_gmres_solve_mixed: bad arguments"); return BG_ERR_ARG; }
  size_t bytes = 16 * (size_t)A->N * nrhs;
  void *dB = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&dB, bytes, stream()));
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = bg_gmres_solve_mixed_device(A, F, P, dB, A->N, nrhs, tol, restart, maxit, inner_tol, stats);
  if (!st) {
    e = cudaMemcpyAsync(B, dB, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(dB, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_gmres_solve_lu_fallback_device(bg_matrix *A, bg_matrix *F, const bg_precond *P, void *dB, int ldb, int nrhs,
                                      double tol, int restart, int maxit, double inner_tol, double *stats) {
  double st4[4] = {0, 0, 0, 0};
  if (!A || !F || !dB || nrhs <= 0 || ldb < A->N) {
    set_error("bg_gmres_solve_lu_fallback: bad arguments");
    return BG_ERR_ARG;
  }
  size_t bytes = 16 * (size_t)A->N * nrhs;
  void *saved = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&saved, bytes, stream()));
  cudaError_t e = cudaMemcpy2DAsync(saved, 16 * (size_t)A->N, dB, 16 * (size_t)ldb, 16 * (size_t)A->N, nrhs,
                                    cudaMemcpyDeviceToDevice, stream());
  int st = e == cudaSuccess ? BG_OK : BG_ERR_CUDA;
  if (st) set_error("gmres fallback: %s", cudaGetErrorString(e));
  if (!st) st = bg_gmres_solve_mixed_device(A, F, P, dB, ldb, nrhs, tol, restart, maxit, inner_tol, st4);
  bool converged = !st && st4[1] <= tol;
  if (!converged && (st == BG_OK || st == BG_ERR_NUMERIC)) {
    // the Krylov solve missed the target: LU of the complex64 copy (tcgen05)
    // and the FP64-refined solve from the original right-hand sides
    e = cudaMemcpy2DAsync(dB, 16 * (size_t)ldb, saved, 16 * (size_t)A->N, 16 * (size_t)A->N, nrhs,
                          cudaMemcpyDeviceToDevice, stream());
    st = e == cudaSuccess ? BG_OK : BG_ERR_CUDA;
    if (st) set_error("gmres fallback: %s", cudaGetErrorString(e));
    if (!st) st = bg_lu_factor(F);
    double rs[3] = {0, 0, 0};
    if (!st) st = bg_lu_solve_refined_device(A, F, dB, ldb, nrhs, tol, 60, rs);
    st4[1] = rs[1];
    st4[3] = 1;
  }
  cudaFreeAsync(saved, stream());
  if (stats) for (int i = 0; i < 4; i++) stats[i] = st4[i];
  return st;
}

int bg_gmres_last_info(double *out) {
  if (!out) { set_error("bg_gmres_last_info: null output"); return BG_ERR_ARG; }
  GmInfo g = gmres_last_info();
  out[0] = g.steps;
  out[1] = g.relres;
  out[2] = g.sweeps;
  out[3] = g.switched;
  out[4] = g.gave_up;
  out[5] = g.longest_cycle;
  return BG_OK;
}

int bg_gmres_solve_lu_fallback(bg_matrix *A, bg_matrix *F, const bg_precond *P, double *B, int nrhs, double tol,
                               int restart, int maxit, double inner_tol, double *stats) {
  if (!A || !B || nrhs <= 0) { set_error("bg_gmres_solve_lu_fallback: bad arguments"); return BG_ERR_ARG; }
  size_t bytes = 16 * (size_t)A->N * nrhs;
  void *dB = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&dB, bytes, stream()));
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = bg_gmres_solve_lu_fallback_device(A, F, P, dB, A->N, nrhs, tol, restart, maxit, inner_tol, stats);
  if (!st) {
    e = cudaMemcpyAsync(B, dB, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(dB, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("gmres: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_lu_solve(bg_matrix *m, double *B, int nrhs) {
  if (!m || !B || nrhs <= 0) { set_error("bg_lu_solve: bad arguments"); return BG_ERR_ARG; }
  if (!m->factored) { set_error("bg_lu_solve: matrix is not LU-factored"); return BG_ERR_STATE; }
  if (m->precision == BG_C64) {
    std::vector<float> h(2 * (size_t)m->N * nrhs);
    for (size_t i = 0; i < h.size(); i++) h[i] = (float)B[i];
    void *d = nullptr;
    BG_CUDA_TRY(cudaMalloc(&d, sizeof(float) * h.size()));
    int st = BG_OK;
    cudaError_t e = cudaMemcpy(d, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
    if (!st) st = bg_lu_solve_device(m, d, m->N, nrhs);
    if (!st) {
      cudaError_t e2 = cudaStreamSynchronize(stream());
      if (e2 == cudaSuccess) e2 = cudaMemcpy(h.data(), d, sizeof(float) * h.size(), cudaMemcpyDeviceToHost);
      if (e2 != cudaSuccess) { set_error("solve: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
    }
    cudaFree(d);
    if (!st) for (size_t i = 0; i < h.size(); i++) B[i] = h[i];
    return st;
  }
  size_t bytes = 16 * (size_t)m->N * nrhs;
  void *dB = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&dB, bytes, stream()));
  int st = BG_OK;
  cudaError_t e = cudaMemcpyAsync(dB, B, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = bg_lu_solve_device(m, dB, m->N, nrhs);
  if (!st) {
    e = cudaMemcpyAsync(B, dB, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(dB, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("solve: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_rhs_planewave_device(bg_geometry *g, double wr, double wi, const double *E0, const double *nhat, void *out) {
  if (!g || !E0 || !nhat || !out) { set_error("bg_rhs_planewave: bad arguments"); return BG_ERR_ARG; }
  if (wr == 0.0 && wi == 0.0) { set_error("bg_rhs_planewave: omega must be nonzero"); return BG_ERR_ARG; }
  int st = upload_geometry(g);
  if (st) return st;
  return rhs_planewave(g, wr, wi, E0, nhat, out);
}

int bg_rhs_planewave(bg_geometry *g, double wr, double wi, const double *E0, const double *nhat, double *out) {
  if (!g || !out) { set_error("bg_rhs_planewave: bad arguments"); return BG_ERR_ARG; }
  int st = upload_geometry(g);
  if (st) return st;
  size_t bytes = 16 * (size_t)g->N;
  void *d = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&d, bytes, stream()));
  st = bg_rhs_planewave_device(g, wr, wi, E0, nhat, d);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(d, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("rhs: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_pft(bg_geometry *g, double wr, double wi, const double *J, const double *E0, const double *nhat, int method,
           double *out) {
  if (!g || !J || !out || (method != BG_PFT_EMT && method != BG_PFT_OVERLAP)) { set_error("bg_pft: bad arguments"); return BG_ERR_ARG; }
  if (method == BG_PFT_EMT && (!E0 || !nhat)) { set_error("bg_pft: EMT needs the incident plane wave"); return BG_ERR_ARG; }
  int st = upload_geometry(g);
  if (st) return st;
  size_t bytes = 16 * (size_t)g->N;
  void *d = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&d, bytes, stream()));
  cudaError_t e = cudaMemcpyAsync(d, J, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = pft(g, wr, wi, d, E0, nhat, method, out);
  cudaFreeAsync(d, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("pft: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_pft_full(bg_geometry *g, double wr, double wi, const double *J, const double *E0, const double *nhat,
                double *out) {
  if (!g || !J || !out || !E0 || !nhat) { set_error("bg_pft_full: bad arguments"); return BG_ERR_ARG; }
  if (wr == 0.0) { set_error("bg_pft_full: the force and torque columns need real(omega) != 0"); return BG_ERR_ARG; }
  int st = upload_geometry(g);
  if (st) return st;
  size_t bytes = 16 * (size_t)g->N;
  void *d = nullptr;
  BG_CUDA_TRY(cudaMallocAsync(&d, bytes, stream()));
  cudaError_t e = cudaMemcpyAsync(d, J, bytes, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = pft_emt_full(g, wr, wi, d, E0, nhat, out);
  cudaFreeAsync(d, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("pft: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

static int fields_args(const char *fn, bg_geometry *g, const double *E0, const double *nhat, int npts,
                       const void *X, const void *out) {
  if (!g || npts < 0 || (npts > 0 && (!X || !out))) { set_error("%s: bad arguments", fn); return BG_ERR_ARG; }
  if (E0 && !nhat) { set_error("%s: the plane wave needs nhat", fn); return BG_ERR_ARG; }
  return BG_OK;
}

int bg_get_fields(bg_geometry *g, double wr, double wi, const double *J, const double *E0, const double *nhat,
                  int npts, const double *X, double *out) {
  int st = fields_args("bg_get_fields", g, E0, nhat, npts, X, out);
  if (st || npts == 0) return st;
  if ((st = upload_geometry(g))) return st;
  size_t jb = J ? 16 * (size_t)g->N : 0, xb = 24 * (size_t)npts, ob = 96 * (size_t)npts;
  char *d = nullptr;
  BG_CUDA_TRY(cudaMallocAsync((void **)&d, jb + xb + ob, stream()));
  void *dJ = J ? d : nullptr;
  double *dX = (double *)(d + jb);
  void *dO = d + jb + xb;
  cudaError_t e = cudaSuccess;
  if (J) e = cudaMemcpyAsync(dJ, J, jb, cudaMemcpyHostToDevice, stream());
  if (e == cudaSuccess) e = cudaMemcpyAsync(dX, X, xb, cudaMemcpyHostToDevice, stream());
  if (e != cudaSuccess) { set_error("H2D: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  if (!st) st = get_fields(g, wr, wi, dJ, E0, E0 ? nhat : nullptr, npts, dX, dO);
  if (!st) {
    e = cudaMemcpyAsync(out, dO, ob, cudaMemcpyDeviceToHost, stream());
    if (e != cudaSuccess) { set_error("D2H: %s", cudaGetErrorString(e)); st = BG_ERR_CUDA; }
  }
  cudaFreeAsync(d, stream());
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("get_fields: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_get_fields_device(bg_geometry *g, double wr, double wi, const void *J_dev, const double *E0,
                         const double *nhat, int npts, const double *X_dev, void *out_dev) {
  int st = fields_args("bg_get_fields_device", g, E0, nhat, npts, X_dev, out_dev);
  if (st || npts == 0) return st;
  st = get_fields(g, wr, wi, J_dev, E0, E0 ? nhat : nullptr, npts, X_dev, out_dev);
  cudaError_t e2 = cudaStreamSynchronize(stream());
  if (!st && e2 != cudaSuccess) { set_error("get_fields: %s", cudaGetErrorString(e2)); st = BG_ERR_CUDA; }
  return st;
}

int bg_zgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc) {
  if (M < 0 || N < 0 || K < 0 || (M && N && K && (!A || !B || !C)) || lda < M || ldb < K || ldc < M ||
      lda < 1 || ldb < 1 || ldc < 1) {
    set_error("bg_zgemm_sub_device: bad arguments");
    return BG_ERR_ARG;
  }
  return zgemm_sub_device(M, N, K, A, lda, B, ldb, C, ldc);
}

int bg_cgemm_sub_device(int M, int N, int K, const void *A, int lda, const void *B, int ldb, void *C, int ldc) {
  if (M < 0 || N < 0 || K < 0 || (M && N && K && (!A || !B || !C)) || lda < M || ldb < K || ldc < M ||
      lda < 1 || ldb < 1 || ldc < 1) {
    set_error("bg_cgemm_sub_device: bad arguments");
    return BG_ERR_ARG;
  }
  int st = ensure_device();
  if (st) return st;
  return cgemm_sub_device(M, N, K, A, lda, B, ldb, C, ldc);
}

long long bg_kernel_launch_count(void) { return g_launches.load(); }

int bg_profile_begin(void) {
  int st = ensure_device();
  if (st) return st;
  for (auto &r : s_recs) { s_pool.push_back(r.a); s_pool.push_back(r.b); }
  s_recs.clear();
  s_prof = true;
  return BG_OK;
}

int bg_profile_read(int n, long long *counts, double *ms, double *flops) {
  if (n <= 0 || !counts || !ms || !flops) { set_error("bg_profile_read: bad arguments"); return BG_ERR_ARG; }
  BG_CUDA_TRY(cudaStreamSynchronize(s_stream));
  for (int i = 0; i < n; i++) { counts[i] = 0; ms[i] = 0; flops[i] = 0; }
  for (auto &r : s_recs) {
    if (r.cls >= n) continue;
    float t = 0;
    BG_CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
    counts[r.cls]++;
    ms[r.cls] += t;
    flops[r.cls] += r.flops;
  }
  return BG_OK;
}

int bg_profile_end(void) {
  s_prof = false;
  return BG_OK;
}

int bg_synchronize(void) {
  int st = ensure_device();
  if (st) return st;
  BG_CUDA_TRY(cudaStreamSynchronize(stream()));
  return BG_OK;
}

void *bg_stream(void) {
  if (ensure_device()) return nullptr;
  return (void *)stream();
}

}  // extern "C"
