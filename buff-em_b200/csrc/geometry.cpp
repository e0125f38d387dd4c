// Host-side geometry of the B200 BUFF-EM path: gmsh reader, face list / SWG
// numbering, .buffgeo parser, structure-of-arrays upload and the near-pair
// lists that route basis-function pairs to the near-field kernels.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace bg {

static double dist3(const double *a, const double *b) {
  double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  return std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
}

// ReadGMSHFile, ReadGMSHFile.cc:66-261: $Nodes/$Elements (gmsh 2.x) or the
// legacy $NOD/$ELM format; node ids remapped; vertices closer than 1e-6 are
// merged onto the lower index (:130-141); only element type 4 (tetrahedron)
// is kept; the one-time transformation is applied before the merge (:124).
static int read_gmsh(Object &o, const char *path, const double *xf) {
  FILE *f = std::fopen(path, "r");
  if (!f) { set_error("cannot open mesh file %s", path); return BG_ERR_IO; }
  char buf[512];
  int legacy = -1;
  while (std::fgets(buf, sizeof buf, f)) {
    if (!std::strncmp(buf, "$Nodes", 6)) { legacy = 0; break; }
    if (!std::strncmp(buf, "$NOD", 4)) { legacy = 1; break; }
  }
  auto fail = [&](const char *msg) { std::fclose(f); set_error("%s: %s", path, msg); return BG_ERR_IO; };
  if (legacy < 0 || !std::fgets(buf, sizeof buf, f)) return fail("no node section");
  int nv = std::atoi(buf);
  if (nv <= 0) return fail("invalid number of nodes");
  std::vector<int> map(2 * (size_t)nv + 1, -1);
  o.nv = nv;
  o.V.assign(3 * (size_t)nv, 0.0);
  for (int i = 0; i < nv; i++) {
    int id;
    if (!std::fgets(buf, sizeof buf, f) ||
        std::sscanf(buf, "%d %lf %lf %lf", &id, &o.V[3 * i], &o.V[3 * i + 1], &o.V[3 * i + 2]) != 4)
      return fail("invalid node specification");
    if (id < 0 || id > 2 * nv) return fail("node id out of range");
    map[id] = i;
  }
  if (xf)
    for (int i = 0; i < nv; i++) {
      double *x = &o.V[3 * i], y[3];
      for (int k = 0; k < 3; k++) y[k] = xf[3 * k] * x[0] + xf[3 * k + 1] * x[1] + xf[3 * k + 2] * x[2] + xf[9 + k];
      for (int k = 0; k < 3; k++) x[k] = y[k];
    }
  for (int i = 0; i < nv; i++)
    for (int j = i + 1; j < nv; j++)
      if (dist3(&o.V[3 * i], &o.V[3 * j]) < 1.0e-6)
        for (size_t g = 0; g < map.size(); g++)
          if (map[g] == j) map[g] = i;
  if (!std::fgets(buf, sizeof buf, f)) return fail("nodes section not terminated");
  if (std::strncmp(buf, legacy ? "$ENDNOD" : "$EndNodes", legacy ? 7 : 9)) return fail("unexpected keyword");
  if (!std::fgets(buf, sizeof buf, f)) return fail("elements section missing");
  if (std::strncmp(buf, legacy ? "$ELM" : "$Elements", legacy ? 4 : 9)) return fail("unexpected keyword");
  if (!std::fgets(buf, sizeof buf, f)) return fail("invalid number of elements");
  int ne = -1;
  if (std::sscanf(buf, "%d", &ne) != 1 || ne < 0) return fail("invalid number of elements");
  o.VI.clear();
  for (int e = 0; e < ne; e++) {
    if (!std::fgets(buf, sizeof buf, f)) return fail("too few elements");
    int num, type, vi[4] = {0, 0, 0, 0};
    if (legacy) {
      int rp, re, nc;
      if (std::sscanf(buf, "%d %d %d %d %d %d %d %d %d", &num, &type, &rp, &re, &nc, vi, vi + 1, vi + 2,
                      vi + 3) < 5)
        return fail("invalid element specification");
    } else {
      int ntags, nr, pos;
      if (std::sscanf(buf, "%d %d %d%n", &num, &type, &ntags, &nr) < 3) return fail("invalid element specification");
      pos = nr;
      for (int t = 0; t < ntags; t++) {
        int dmy;
        if (std::sscanf(buf + pos, "%d%n", &dmy, &nr) != 1) return fail("invalid element tags");
        pos += nr;
      }
      int nc = std::sscanf(buf + pos, "%d %d %d %d", vi, vi + 1, vi + 2, vi + 3);
      if (type == 4 && nc != 4) return fail("invalid tetrahedron specification");
    }
    if (type == 4) {
      for (int k = 0; k < 4; k++) {
        if (vi[k] < 0 || vi[k] > 2 * nv || map[vi[k]] < 0) return fail("tetrahedron references unknown node");
        o.VI.push_back(map[vi[k]]);
      }
    }
  }
  std::fclose(f);
  o.nt = (int)(o.VI.size() / 4);
  if (o.nt == 0) { set_error("%s: no tetrahedra found", path); return BG_ERR_IO; }
  // NewSWGTet, SWGVolume.cc:50-85: signed volume (1/6) A.(BxC)
  o.vol.resize(o.nt);
  for (int t = 0; t < o.nt; t++) {
    const double *V1 = &o.V[3 * o.VI[4 * t]], *V2 = &o.V[3 * o.VI[4 * t + 1]];
    const double *V3 = &o.V[3 * o.VI[4 * t + 2]], *V4 = &o.V[3 * o.VI[4 * t + 3]];
    double A[3], B[3], C[3];
    for (int i = 0; i < 3; i++) { A[i] = V2[i] - V1[i]; B[i] = V3[i] - V1[i]; C[i] = V4[i] - V1[i]; }
    o.vol[t] = (A[0] * (B[1] * C[2] - B[2] * C[1]) + A[1] * (B[2] * C[0] - B[0] * C[2]) +
                A[2] * (B[0] * C[1] - B[1] * C[0])) / 6.0;
  }
  return BG_OK;
}

// InitFaceList, InitFaceList.cc:69-279.  Faces are keyed by their sorted
// vertex triple in per-minimum-vertex lists; the first tetrahedron to visit a
// face is its P side, the second its M side, and the interior index is given
// on the second visit -- this fixes the matrix row order.  Exterior faces are
// numbered after the interior ones in list order (most recent first).
static int init_faces(Object &o) {
  std::vector<std::vector<int>> lists(o.nv);
  std::vector<Face> all;
  all.reserve(2 * (size_t)o.nt + 16);
  o.nif = 0;
  for (int nt = 0; nt < o.nt; nt++)
    for (int nf = 0; nf < 4; nf++) {
      const int *T = &o.VI[4 * nt];
      int VI[3] = {T[(nf + 1) % 4], T[(nf + 2) % 4], T[(nf + 3) % 4]};
      int iMin = 0, iMax = 0;
      if (VI[1] < VI[iMin]) iMin = 1;
      if (VI[2] < VI[iMin]) iMin = 2;
      if (VI[1] > VI[iMax]) iMax = 1;
      if (VI[2] > VI[iMax]) iMax = 2;
      int vmin = VI[iMin], vmid = VI[3 - iMin - iMax], vmax = VI[iMax];
      int iQ = T[nf];
      int found = -1;
      for (int k = (int)lists[vmin].size() - 1; k >= 0; k--) {
        const Face &F = all[lists[vmin][k]];
        if (F.iV2 == vmid && F.iV3 == vmax) { found = lists[vmin][k]; break; }
      }
      if (found >= 0) {
        Face &F = all[found];
        if (F.iMTet != -1) {
          set_error("%s: invalid mesh topology: face %d of tet %d also belongs to tets %d and %d",
                    o.meshfile.c_str(), nf, nt, F.iPTet, F.iMTet);
          return BG_ERR_TOPOLOGY;
        }
        F.iQM = iQ; F.iMTet = nt; F.MIndex = nf; F.Index = o.nif++;
        const double *V = o.V.data();
        F.radius = dist3(F.cen, V + 3 * F.iQP);
        F.radius = std::fmax(F.radius, dist3(F.cen, V + 3 * F.iV1));
        F.radius = std::fmax(F.radius, dist3(F.cen, V + 3 * F.iV2));
        F.radius = std::fmax(F.radius, dist3(F.cen, V + 3 * F.iV3));
        F.radius = std::fmax(F.radius, dist3(F.cen, V + 3 * F.iQM));
      } else {
        Face F{};
        F.iV1 = vmin; F.iV2 = vmid; F.iV3 = vmax; F.iQP = iQ; F.iQM = -1;
        F.iPTet = nt; F.iMTet = -1; F.PIndex = nf; F.MIndex = -1; F.Index = -1;
        const double *V1 = &o.V[3 * vmin], *V2 = &o.V[3 * vmid], *V3 = &o.V[3 * vmax];
        double A[3], B[3];
        for (int i = 0; i < 3; i++) {
          F.cen[i] = (V1[i] + V2[i] + V3[i]) / 3.0;
          A[i] = V2[i] - V1[i]; B[i] = V3[i] - V1[i];
        }
        double c0 = A[1] * B[2] - A[2] * B[1], c1 = A[2] * B[0] - A[0] * B[2], c2 = A[0] * B[1] - A[1] * B[0];
        F.area = 0.5 * std::sqrt(c0 * c0 + c1 * c1 + c2 * c2);
        F.radius = 0.0;
        lists[vmin].push_back((int)all.size());
        all.push_back(F);
      }
    }
  o.ntf = (int)all.size();
  o.F.assign(o.ntf, Face{});
  o.FI.assign(4 * (size_t)o.nt, -1);
  int next = 0;
  for (int v = 0; v < o.nv; v++)
    for (int k = (int)lists[v].size() - 1; k >= 0; k--) {
      Face &F = all[lists[v][k]];
      if (F.Index == -1) F.Index = o.nif + next++;
      o.F[F.Index] = F;
      o.FI[4 * F.iPTet + F.PIndex] = F.Index;
      if (F.iMTet != -1) o.FI[4 * F.iMTet + F.MIndex] = F.Index;
    }
  return BG_OK;
}

int load_object(Object &o, const char *meshfile, const double *xf) {
  static const double eye[12] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0};
  if (xf && !std::memcmp(xf, eye, sizeof eye)) xf = nullptr;   // untransformed: nodes as read
  o.meshfile = meshfile;
  int st = read_gmsh(o, meshfile, xf);
  if (st) return st;
  if (xf) for (int k = 0; k < 3; k++) o.origin[k] = xf[9 + k];
  return init_faces(o);
}

int refresh_materials(bg_geometry *g, double wr, double wi) {
  if (!g->dispersive) return BG_OK;
  std::vector<bg_material> mats(g->objs.size());
  for (size_t i = 0; i < g->objs.size(); i++) {
    Object &o = g->objs[i];
    if (o.matprop) {
      o.mat = bg_material{};
      o.mat.kind = BG_MAT_CONST_ISO;
      matprop_eps(*o.matprop, wr, wi, o.mat.eps);
    } else if (o.svt && svtensor_position_dependent(*o.svt)) {
      // the program at this Omega: w, the constants and Eps1-3 folded in
      o.mat = bg_material{};
      o.mat.kind = BG_MAT_EXPR;
      if (!g->dev.expr) { set_error("compiled SVTENSOR programs are not on the device"); return BG_ERR_STATE; }
      DevExpr prog{};
      int st = svtensor_compile(*o.svt, wr, wi, &prog);
      if (st) return st;
      // synchronous from pageable memory: prog may leave scope at once
      BG_CUDA_TRY(cudaMemcpy(g->dev.expr + i, &prog, sizeof(DevExpr), cudaMemcpyHostToDevice));
    } else if (o.svt) {
      const double x0[3] = {0.0, 0.0, 0.0};   // position-independent by construction
      o.mat = bg_material{};
      o.mat.kind = BG_MAT_CONST_TENSOR;
      svtensor_eval(*o.svt, wr, wi, x0, o.mat.eps);
    }
    mats[i] = o.mat;
  }
  if (g->dev.mats)   // pageable source: the call returns once the bytes are staged
    BG_CUDA_TRY(cudaMemcpyAsync(g->dev.mats, mats.data(), sizeof(bg_material) * mats.size(), cudaMemcpyHostToDevice,
                                stream()));
  return BG_OK;
}

// ------------------------------------------------------------- device upload
template <class T>
static int dupload(T **dst, const std::vector<T> &src) {
  size_t bytes = sizeof(T) * std::max<size_t>(src.size(), 1);
  BG_CUDA_TRY(cudaMalloc((void **)dst, bytes));
  if (!src.empty()) BG_CUDA_TRY(cudaMemcpy(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice));
  return BG_OK;
}

int upload_geometry(bg_geometry *g) {
  if (g->uploaded) return BG_OK;
  int st = ensure_device();
  if (st) return st;
  std::vector<double> V4, tetP4, tetVol, area, radius, origin;
  std::vector<int4> tetVI, bfV;
  std::vector<int> tetObj;
  std::vector<int2> bfTet, bfQ, bfLoc;
  std::vector<int4> tetFI;
  std::vector<bg_material> mats;
  // 4-point rule (TetCR.cc:35-40): the S31 orbit with a = 0.1381966..., b = 1-3a
  const double qa = 0.13819660112501051, qb = 0.58541019662496850;
  for (size_t no = 0; no < g->objs.size(); no++) {
    const Object &o = g->objs[no];
    int vo = g->vOffset[no], to = g->tOffset[no];
    for (int v = 0; v < o.nv; v++) {
      V4.push_back(o.V[3 * v]); V4.push_back(o.V[3 * v + 1]); V4.push_back(o.V[3 * v + 2]); V4.push_back(0.0);
    }
    for (int t = 0; t < o.nt; t++) {
      const int *T = &o.VI[4 * t];
      tetVI.push_back(make_int4(T[0] + vo, T[1] + vo, T[2] + vo, T[3] + vo));
      tetVol.push_back(o.vol[t]);
      tetObj.push_back((int)no);
      int fi[4];
      for (int k = 0; k < 4; k++) {
        int f = o.FI[4 * t + k];
        fi[k] = (f >= 0 && f < o.nif) ? f + g->bfOffset[no] : -1;
      }
      tetFI.push_back(make_int4(fi[0], fi[1], fi[2], fi[3]));
      double cen[3] = {0, 0, 0};
      for (int i = 0; i < 4; i++)
        for (int k = 0; k < 3; k++) cen[k] += 0.25 * o.V[3 * T[i] + k];
      for (int j = 0; j < 4; j++) {
        double d2 = 0.0;
        for (int k = 0; k < 3; k++) {
          double s = 0.0;
          for (int i = 0; i < 4; i++) s += (i == j ? qb : qa) * o.V[3 * T[i] + k];
          tetP4.push_back(s);
          d2 += (s - cen[k]) * (s - cen[k]);
        }
        tetP4.push_back(0.0);
        g->rule_rmax = std::max(g->rule_rmax, std::sqrt(d2));
      }
    }
    for (int a = 0; a < o.nif; a++) {
      const Face &F = o.F[a];
      bfTet.push_back(make_int2(F.iPTet + to, F.iMTet + to));
      bfQ.push_back(make_int2(F.iQP + vo, F.iQM + vo));
      bfLoc.push_back(make_int2(F.PIndex, F.MIndex));
      bfV.push_back(make_int4(F.iV1 + vo, F.iV2 + vo, F.iV3 + vo, (int)no));
      area.push_back(F.area);
      radius.push_back(F.radius);
    }
    mats.push_back(o.mat);
    for (int k = 0; k < 3; k++) origin.push_back(o.origin[k]);
  }
  // far-field tiles: distinct tetrahedra of each run of BG_FAR_TILE basis functions
  int ntile = (g->N + BG_FAR_TILE - 1) / BG_FAR_TILE;
  std::vector<int> tileTet((size_t)ntile * BG_FAR_TILE_TETS, -1), tileNT(ntile, 0);
  std::vector<int2> bfTileLoc(g->N);
  for (int t = 0; t < ntile; t++) {
    int *list = tileTet.data() + (size_t)t * BG_FAR_TILE_TETS;
    int cnt = 0;
    auto slot = [&](int tet) {
      for (int i = 0; i < cnt; i++)
        if (list[i] == tet) return i;
      list[cnt] = tet;
      return cnt++;
    };
    for (int a = t * BG_FAR_TILE; a < std::min(g->N, (t + 1) * BG_FAR_TILE); a++) {
      int lp = slot(bfTet[a].x);
      int lm = slot(bfTet[a].y);
      bfTileLoc[a] = make_int2(lp, lm);
    }
    tileNT[t] = cnt;
  }
  DevGeom &d = g->dev;
  d.N = g->N; d.NT = g->NT; d.NV = g->NV;
  if ((st = dupload(&d.tileTet, tileTet)) || (st = dupload(&d.tileNT, tileNT)) || (st = dupload(&d.bfTileLoc, bfTileLoc)))
    return st;
  if ((st = dupload(&d.V4, V4)) || (st = dupload(&d.tetVI, tetVI)) || (st = dupload(&d.tetVol, tetVol)) ||
      (st = dupload(&d.tetP4, tetP4)) || (st = dupload(&d.tetObj, tetObj)) || (st = dupload(&d.bfTet, bfTet)) ||
      (st = dupload(&d.bfQ, bfQ)) || (st = dupload(&d.bfLoc, bfLoc)) || (st = dupload(&d.tetFI, tetFI)) || (st = dupload(&d.bfV, bfV)) || (st = dupload(&d.bfArea, area)) ||
      (st = dupload(&d.bfRadius, radius)) || (st = dupload(&d.mats, mats)) || (st = dupload(&d.objOrigin, origin)))
    return st;
  bool any_expr = false;
  for (const Object &o : g->objs) any_expr = any_expr || o.mat.kind == BG_MAT_EXPR;
  if (any_expr) {
    BG_CUDA_TRY(cudaMalloc((void **)&d.expr, sizeof(DevExpr) * g->objs.size()));
    BG_CUDA_TRY(cudaMemset(d.expr, 0, sizeof(DevExpr) * g->objs.size()));
  }
  g->uploaded = true;
  return BG_OK;
}

// ------------------------------------------------------------- near lists
// Near basis-function pairs are the same-object pairs with at least one common
// vertex among {QP, V1, V2, V3, QM} (CompareBFs, SWGVolume.cc:295-344); they take
// the desingularised kernel plus the cached static integrals
// (GMatrixElements.cc:400-420).  Their 4 tetrahedron pairs are collected into a
// list of distinct pairs, split into regular ones (<= 1 common vertex: 16x16
// rule, GMatrixElements.cc:329-341) and singular ones (2..4 common vertices).
int build_near_lists(bg_geometry *g) {
  NearData &nd = g->near;
  if (nd.pairs) return BG_OK;
  int N = g->N;
  std::vector<int> bfobj(N), qp(N), qm(N), v1(N), v2(N), v3(N), tp(N), tm(N);
  for (size_t no = 0; no < g->objs.size(); no++) {
    const Object &o = g->objs[no];
    int vo = g->vOffset[no], to = g->tOffset[no], bo = g->bfOffset[no];
    for (int a = 0; a < o.nif; a++) {
      const Face &F = o.F[a];
      bfobj[bo + a] = (int)no;
      qp[bo + a] = F.iQP + vo; qm[bo + a] = F.iQM + vo;
      v1[bo + a] = F.iV1 + vo; v2[bo + a] = F.iV2 + vo; v3[bo + a] = F.iV3 + vo;
      tp[bo + a] = F.iPTet + to; tm[bo + a] = F.iMTet + to;
    }
  }
  // vertex -> basis functions touching it
  std::vector<int> cnt(g->NV + 1, 0);
  for (int a = 0; a < N; a++) { cnt[qp[a]]++; cnt[qm[a]]++; cnt[v1[a]]++; cnt[v2[a]]++; cnt[v3[a]]++; }
  std::vector<int> start(g->NV + 1, 0);
  for (int v = 0; v < g->NV; v++) start[v + 1] = start[v] + cnt[v];
  std::vector<int> fill(start.begin(), start.end() - 1), inc(start[g->NV]);
  for (int a = 0; a < N; a++) {
    int vs[5] = {qp[a], v1[a], v2[a], v3[a], qm[a]};
    for (int k = 0; k < 5; k++) inc[fill[vs[k]]++] = a;
  }
  std::vector<int2> pairs;
  std::vector<int> mark(N, -1);
  for (int a = 0; a < N; a++) {
    int vs[5] = {qp[a], v1[a], v2[a], v3[a], qm[a]};
    std::vector<int> row;
    for (int k = 0; k < 5; k++)
      for (int i = start[vs[k]]; i < start[vs[k] + 1]; i++) {
        int b = inc[i];
        if (b >= a && mark[b] != a) { mark[b] = a; row.push_back(b); }
      }
    std::sort(row.begin(), row.end());
    for (int b : row) pairs.push_back(make_int2(a, b));
  }
  // distinct tetrahedron pairs
  std::vector<int> tvi(4 * (size_t)g->NT);
  for (size_t no = 0; no < g->objs.size(); no++) {
    const Object &o = g->objs[no];
    for (int t = 0; t < o.nt; t++)
      for (int k = 0; k < 4; k++) tvi[4 * (size_t)(t + g->tOffset[no]) + k] = o.VI[4 * t + k] + g->vOffset[no];
  }
  std::unordered_map<uint64_t, int> key2tp;
  key2tp.reserve(pairs.size() * 2);
  std::vector<int2> tps;
  std::vector<int4> pairTP(pairs.size());
  for (size_t k = 0; k < pairs.size(); k++) {
    int a = pairs[k].x, b = pairs[k].y;
    int ta[2] = {tp[a], tm[a]}, tb[2] = {tp[b], tm[b]};
    int idx[4];
    for (int sa = 0; sa < 2; sa++)
      for (int sb = 0; sb < 2; sb++) {
        // ordered (row tetrahedron, column tetrahedron): the angular rule of
        // the singular integrals follows the row tetrahedron's vertex order
        // (CompareTets, SWGVolume.cc:357-400), so (x,y) and (y,x) are distinct
        int x = ta[sa], y = tb[sb];
        uint64_t key = ((uint64_t)(uint32_t)x << 32) | (uint32_t)y;
        auto it = key2tp.find(key);
        int id;
        if (it == key2tp.end()) { id = (int)tps.size(); key2tp.emplace(key, id); tps.push_back(make_int2(x, y)); }
        else id = it->second;
        idx[2 * sa + sb] = id;
      }
    pairTP[k] = make_int4(idx[0], idx[1], idx[2], idx[3]);
  }
  // classify and order: regular first, then singular by decreasing cost (c=2,3,4)
  int ntp = (int)tps.size();
  std::vector<int> common(ntp);
  for (int i = 0; i < ntp; i++) {
    int c = 0;
    for (int x = 0; x < 4; x++)
      for (int y = 0; y < 4; y++) c += tvi[4 * (size_t)tps[i].x + x] == tvi[4 * (size_t)tps[i].y + y];
    common[i] = c;
  }
  std::vector<int> order(ntp);
  for (int i = 0; i < ntp; i++) order[i] = i;
  auto rank = [&](int i) { int c = common[i]; return c <= 1 ? 0 : c - 1; };
  std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return rank(i) < rank(j); });
  std::vector<int> newid(ntp);
  for (int i = 0; i < ntp; i++) newid[order[i]] = i;
  std::vector<int4> tpl(ntp), ordA(ntp), ordB(ntp);
  int nreg = 0;
  for (int i = 0; i < ntp; i++) {
    int o = order[i];
    int A = tps[o].x, B = tps[o].y, c = common[o];
    if (c <= 1) nreg++;
    tpl[i] = make_int4(A, B, c, 0);
    // CompareTets (SWGVolume.cc:357-400): common vertices first in A's order
    const int *VA = &tvi[4 * (size_t)A], *VB = &tvi[4 * (size_t)B];
    bool ca[4] = {false, false, false, false}, cb[4] = {false, false, false, false};
    for (int x = 0; x < 4; x++)
      for (int y = 0; y < 4; y++)
        if (VA[x] == VB[y]) ca[x] = cb[y] = true;
    int oa[4], ob[4], na = 0, nb = 0;
    for (int x = 0; x < 4; x++) if (ca[x]) { oa[na++] = VA[x]; ob[nb++] = VA[x]; }
    for (int x = 0; x < 4; x++) { if (!ca[x]) oa[na++] = VA[x]; if (!cb[x]) ob[nb++] = VB[x]; }
    ordA[i] = make_int4(oa[0], oa[1], oa[2], oa[3]);
    ordB[i] = make_int4(ob[0], ob[1], ob[2], ob[3]);
  }
  for (auto &p : pairTP) {
    int *q = &p.x;
    for (int j = 0; j < 4; j++) q[j] = newid[q[j] & ~(1 << 30)] | (q[j] & (1 << 30));
  }
  nd.npairs = (int)pairs.size();
  nd.ntp = ntp;
  nd.ntp_reg = nreg;
  for (int i = 0; i < ntp; i++)
    if (common[i] >= 2) nd.nsing_c[std::min(common[i], 4) - 2]++;
  int st;
  if ((st = dupload(&nd.pairs, pairs)) || (st = dupload(&nd.pairTP, pairTP)) || (st = dupload(&nd.tp, tpl)) ||
      (st = dupload(&nd.tpOrdA, ordA)) || (st = dupload(&nd.tpOrdB, ordB)))
    return st;
  BG_CUDA_TRY(cudaMalloc(&nd.fibbi, sizeof(double) * 6 * std::max(1, nd.npairs)));
  BG_CUDA_TRY(cudaMalloc(&nd.tpMom, sizeof(double) * 24 * std::max(1, ntp)));
  return BG_OK;
}

// ------------------------------------------------------------- .buffgeo
static bool parse_complex(const char *s, double *re, double *im) {
  // forms: 10, 4+0.2i, 4-0.2i, 4+0.2j, 0.2i
  char *end;
  double a = std::strtod(s, &end);
  if (end == s) return false;
  if ((*end == 'i' || *end == 'j' || *end == 'I') && end[1] == 0) { *re = 0; *im = a; return true; }
  if (*end == 0) { *re = a; *im = 0; return true; }
  const char *p = end;
  double b = std::strtod(p, &end);
  if (end == p || (*end != 'i' && *end != 'j' && *end != 'I') || end[1] != 0) return false;
  *re = a; *im = b;
  return true;
}

// ------------------------------------------------ one-time transformations
// XP = M X + D with xf = (M row-major, D): the GTransformation of SCUFF-EM's
// libhrutil, which the reference links but does not ship.  A later
// transformation G is composed after the running one (OTGT->Transform(G),
// SWGGeometry.cc:111-121): M <- M_G M, D <- M_G D + D_G.
static void xf_identity(double xf[12]) {
  for (int k = 0; k < 12; k++) xf[k] = 0.0;
  xf[0] = xf[4] = xf[8] = 1.0;
}

static void xf_compose(double xf[12], const double g[12]) {
  double r[12];
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++)
      r[3 * i + j] = g[3 * i] * xf[j] + g[3 * i + 1] * xf[3 + j] + g[3 * i + 2] * xf[6 + j];
    r[9 + i] = g[3 * i] * xf[9] + g[3 * i + 1] * xf[10] + g[3 * i + 2] * xf[11] + g[9 + i];
  }
  for (int k = 0; k < 12; k++) xf[k] = r[k];
}

static bool parse_real(const std::string &t, double *v) {
  if (t.empty()) return false;
  char *end;
  *v = std::strtod(t.c_str(), &end);
  return *end == 0;
}

static std::string upper_case(std::string s) {
  for (auto &c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// t equals a (or b), ignoring the case of t; a and b are upper case
static bool keyword_is(const std::string &t, const char *a, const char *b = nullptr) {
  std::string U = upper_case(t);
  return U == a || (b && U == b);
}

// Parses tok[0..] as a sequence of "DISPLACED dx dy dz" and
// "ROTATED theta ABOUT ax ay az" (theta in degrees, right-handed about the
// axis through the origin; DISP and ROT are accepted as short forms),
// composing each onto xf in order.  The whole line must be consumed (the
// reference's "junk at end of line", SWGGeometry.cc:122-126).
static bool parse_transforms(const std::vector<std::string> &tok, double xf[12], std::string &err) {
  size_t t = 0;
  while (t < tok.size()) {
    double g[12];
    xf_identity(g);
    if (keyword_is(tok[t], "DISPLACED", "DISP")) {
      if (t + 4 > tok.size()) { err = "DISPLACED needs three numbers"; return false; }
      for (int k = 0; k < 3; k++)
        if (!parse_real(tok[t + 1 + k], &g[9 + k])) { err = "bad number " + tok[t + 1 + k]; return false; }
      t += 4;
    } else if (keyword_is(tok[t], "ROTATED", "ROT")) {
      double th, a[3];
      if (t + 6 > tok.size() || !keyword_is(tok[t + 2], "ABOUT")) { err = "ROTATED needs: angle ABOUT ax ay az"; return false; }
      if (!parse_real(tok[t + 1], &th)) { err = "bad angle " + tok[t + 1]; return false; }
      for (int k = 0; k < 3; k++)
        if (!parse_real(tok[t + 3 + k], &a[k])) { err = "bad number " + tok[t + 3 + k]; return false; }
      double n = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      if (!(n > 0)) { err = "rotation axis is zero"; return false; }
      for (int k = 0; k < 3; k++) a[k] /= n;
      // Rodrigues: R = cos I + sin [a]x + (1 - cos) a a^T
      double c = std::cos(th * M_PI / 180.0), sn = std::sin(th * M_PI / 180.0);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) g[3 * i + j] = (1.0 - c) * a[i] * a[j] + (i == j ? c : 0.0);
      g[1] -= sn * a[2]; g[2] += sn * a[1];
      g[3] += sn * a[2]; g[5] -= sn * a[0];
      g[6] -= sn * a[1]; g[7] += sn * a[0];
      t += 6;
    } else {
      err = t ? "junk at end of line" : "unknown transformation " + tok[t];
      return false;
    }
    xf_compose(xf, g);
  }
  return true;
}

// ------------------------------------------------------------- .buffgeo
static std::vector<std::string> tokenize(const char *line) {
  std::vector<std::string> tok;
  const char *p = line;
  while (*p) {
    while (*p && std::isspace((unsigned char)*p)) p++;
    const char *q = p;
    while (*q && !std::isspace((unsigned char)*q)) q++;
    if (q > p) tok.emplace_back(p, q);
    p = q;
  }
  return tok;
}

// one whole line of f (any length), without its newline
static bool get_line(FILE *f, std::string &line) {
  line.clear();
  char buf[1024];
  while (std::fgets(buf, sizeof buf, f)) {
    line += buf;
    if (!line.empty() && line.back() == '\n') { line.pop_back(); return true; }
  }
  return !line.empty();
}

static bool readable(const std::string &f) {
  FILE *t = std::fopen(f.c_str(), "r");
  if (t) std::fclose(t);
  return t != nullptr;
}

// Mesh files named by a relative path are looked up in the directory of the
// .buffgeo file, then in each directory of BUFF_MESH_PATH (colon-separated,
// the reference's search path, SWGVolume.cc:101-107), then in each MESHPATH
// directory of the file (SWGGeometry.cc:276-292, relative ones taken from the
// .buffgeo file's directory), then in the working directory.
static std::string find_file(const std::string &fn, const std::string &dir, const char *env,
                             const std::vector<std::string> &meshpath) {
  if (fn.empty() || fn[0] == '/') return fn;
  std::vector<std::string> cand{dir + "/" + fn};
  if (const char *mp = std::getenv(env)) {
    std::string s = mp;
    size_t a = 0;
    while (a <= s.size()) {
      size_t b = s.find(':', a);
      if (b == std::string::npos) b = s.size();
      if (b > a) cand.push_back(s.substr(a, b - a) + "/" + fn);
      a = b + 1;
    }
  }
  for (auto &d : meshpath) cand.push_back(d + "/" + fn);
  cand.push_back(fn);
  for (auto &c : cand)
    if (readable(c)) return c;
  return cand[0];
}

static std::string find_mesh(const std::string &fn, const std::string &dir, const std::vector<std::string> &meshpath) {
  return find_file(fn, dir, "BUFF_MESH_PATH", meshpath);
}

// MATERIAL argument: CONST_EPS_<complex> or VACUUM; other names refer to
// MATERIAL ... ENDMATERIAL sections of the file (matprop.cpp).  SVTENSOR files
// may depend on frequency and on position: position-dependent ones are
// compiled at each frequency into device programs (BG_MAT_EXPR).
static bool parse_material(const std::string &M, bg_material &m) {
  std::string U = M;
  for (auto &c : U) c = (char)std::toupper((unsigned char)c);
  m = bg_material{};
  m.kind = BG_MAT_CONST_ISO;
  if (U.rfind("CONST_EPS_", 0) == 0) return parse_complex(M.c_str() + 10, &m.eps[0], &m.eps[1]);
  if (U == "VACUUM") { m.eps[0] = 1.0; m.eps[1] = 0.0; return true; }
  return false;
}

static int parse_object_lines(const std::vector<std::vector<std::string>> &lines, const std::vector<int> &lineno,
                              int endline, const char *path, const std::string &dir,
                              const std::vector<std::string> &meshpath, MatDB &db, GeoObject &o) {
  bool have_mesh = false, have_mat = false;
  std::string err;
  for (size_t l = 0; l < lines.size(); l++) {
    const auto &tok = lines[l];
    if (keyword_is(tok[0], "MESHFILE")) {
      if (tok.size() != 2) err = "MESHFILE keyword requires one argument";
      else { o.mesh = find_mesh(tok[1], dir, meshpath); have_mesh = true; }
    } else if (keyword_is(tok[0], "MATERIAL", "SVTENSOR")) {
      if (tok.size() != 2) err = tok[0] + " keyword requires one argument";
      else if (keyword_is(tok[0], "SVTENSOR")) {
        // SVTensor.cc:41-84: looked up along BUFF_SVTENSOR_PATH
        std::shared_ptr<const SVTensorFn> t;
        std::string file = find_file(tok[1], dir, "BUFF_SVTENSOR_PATH", {});
        if (svtensor_parse_file(file, db, t)) return BG_ERR_IO;
        o.svt = t;
        o.matprop.reset();
        o.mat = bg_material{};
        if (svtensor_position_dependent(*t)) {
          // evaluated on the device from a program compiled at each Omega
          o.mat.kind = BG_MAT_EXPR;
        } else {
          o.mat.kind = BG_MAT_CONST_TENSOR;
          const double x0[3] = {0.0, 0.0, 0.0};
          svtensor_eval(*t, 1.0, 0.0, x0, o.mat.eps);   // replaced by the tensor at Omega before every use
        }
        have_mat = true;
      }
      else if (parse_material(tok[1], o.mat)) { o.matprop.reset(); o.svt.reset(); have_mat = true; }
      else if (keyword_is(tok[1].substr(0, std::min<size_t>(10, tok[1].size())), "CONST_EPS_"))
        err = "bad permittivity " + tok[1];
      else {
        // the latest MATERIAL section of that name, ignoring case (as the
        // MatProp database is searched)
        for (size_t k = db.size(); k-- > 0 && !have_mat;)
          if (keyword_is(tok[1], upper_case(db[k].first).c_str())) {
            o.matprop = db[k].second;
            o.svt.reset();
            o.mat = bg_material{};
            o.mat.kind = BG_MAT_CONST_ISO;
            matprop_eps(*o.matprop, 1.0, 0.0, o.mat.eps);   // replaced by eps(Omega) before every use
            have_mat = true;
          }
        if (!have_mat)
          err = "unknown material " + tok[1] + " (CONST_EPS_<value>, VACUUM or a MATERIAL section above)";
      }
    } else if (keyword_is(tok[0], "DISPLACED") || keyword_is(tok[0], "ROTATED")) {
      parse_transforms(tok, o.xf, err);
    } else {
      err = "syntax error";
    }
    if (!err.empty()) { set_error("%s:%d: %s", path, lineno[l], err.c_str()); return BG_ERR_IO; }
  }
  if (!have_mesh) { set_error("%s:%d: no MESHFILE specified for object", path, endline); return BG_ERR_IO; }
  if (!have_mat) { set_error("%s:%d: no MATERIAL or SVTENSOR specified for object", path, endline); return BG_ERR_IO; }
  return BG_OK;
}

// A name MESH__<mesh>[__MAT__<material>] stands for a one-object geometry
// with MESHFILE <mesh>.vmsh (extension of <mesh> dropped) and that material
// (SWGGeometry.cc:167-209; the reference writes it out as a .buffgeo file,
// here it is parsed in memory).
static bool special_name(const char *path, std::vector<std::vector<std::string>> &lines) {
  std::string s = path;
  if (s.size() < 7 || s.compare(0, 6, "MESH__")) return false;
  s = s.substr(6);
  std::string mat, svt;
  size_t pm = s.find("__MAT__"), ps = s.find("__SVT__");
  if (pm != std::string::npos) mat = s.substr(pm + 7, ps != std::string::npos && ps > pm ? ps - pm - 7 : std::string::npos);
  if (ps != std::string::npos) svt = s.substr(ps + 7, pm != std::string::npos && pm > ps ? pm - ps - 7 : std::string::npos);
  std::string mesh = s.substr(0, std::min(pm, ps));
  size_t slash = mesh.find_last_of('/'), dot = mesh.find_last_of('.');
  if (dot != std::string::npos && (slash == std::string::npos || dot > slash)) mesh = mesh.substr(0, dot);
  lines.push_back({"MESHFILE", mesh + ".vmsh"});
  if (pm != std::string::npos) lines.push_back({"MATERIAL", mat});
  if (ps != std::string::npos) lines.push_back({"SVTENSOR", svt + ".SVTensor"});
  return true;
}

// ------------------------------------------------------- .trans files
// A list of geometrical transformations (SCUFF-EM's GTComplex list, read by
// ReadTransFile; used by buff-neq's --TransFile, CreateBNEQData.cc:58-66):
//   TRANS <tag> OBJECT <label> DISP dx dy dz [ROT theta ABOUT ax ay az ...]
//               [OBJECT <label> ...]
// on one line, or TRANS <tag> on its own line followed by OBJECT lines and
// ENDTRANS.  Objects not named keep their position.
static int parse_trans_tokens(const std::vector<std::string> &tok, size_t t, TransEntry &e, std::string &err) {
  while (t < tok.size()) {
    if (!keyword_is(tok[t], "OBJECT", "SURFACE")) { err = "expected OBJECT <label>, got " + tok[t]; return BG_ERR_IO; }
    if (t + 1 >= tok.size()) { err = "OBJECT needs a label"; return BG_ERR_IO; }
    std::string label = tok[t + 1];
    size_t u = t + 2;
    while (u < tok.size() && !keyword_is(tok[u], "OBJECT", "SURFACE")) u++;
    std::vector<std::string> ops(tok.begin() + (long)t + 2, tok.begin() + (long)u);
    if (ops.empty()) { err = "no transformation given for object " + label; return BG_ERR_IO; }
    TransEntry::Op op;
    op.label = label;
    xf_identity(op.xf);
    if (!parse_transforms(ops, op.xf, err)) return BG_ERR_IO;
    e.ops.push_back(op);
    t = u;
  }
  return BG_OK;
}

int parse_trans_file(const char *path, std::vector<TransEntry> &out) {
  FILE *f = std::fopen(path, "r");
  if (!f) { set_error("could not open %s", path); return BG_ERR_IO; }
  std::string buf;
  int lineno = 0, start = 0;
  bool open = false;
  TransEntry cur;
  std::string err;
  auto fail = [&](int ln) {
    std::fclose(f);
    set_error("%s:%d: %s", path, ln, err.c_str());
    return BG_ERR_IO;
  };
  while (get_line(f, buf)) {
    lineno++;
    std::vector<std::string> tok = tokenize(buf.c_str());
    if (tok.empty() || tok[0][0] == '#') continue;
    if (open) {
      if (keyword_is(tok[0], "ENDTRANS")) {
        out.push_back(cur);
        open = false;
      } else if (parse_trans_tokens(tok, 0, cur, err)) {
        return fail(lineno);
      }
    } else if (keyword_is(tok[0], "TRANS")) {
      if (tok.size() < 2) { err = "TRANS needs a tag"; return fail(lineno); }
      cur = TransEntry{};
      cur.tag = tok[1];
      if (tok.size() == 2) {
        open = true;
        start = lineno;
      } else {
        if (parse_trans_tokens(tok, 2, cur, err)) return fail(lineno);
        out.push_back(cur);
      }
    } else {
      err = "syntax error";
      return fail(lineno);
    }
  }
  std::fclose(f);
  if (open) { set_error("%s:%d: TRANS without ENDTRANS", path, start); return BG_ERR_IO; }
  if (out.empty()) { set_error("%s: no transformations", path); return BG_ERR_IO; }
  return BG_OK;
}

// SWGGeometry::Transform (SWGGeometry.cc:426-439, SWGVolume.cc:208-236): each
// named object's transformation is applied after its one-time one.
int apply_trans(const TransEntry &e, std::vector<GeoObject> &objs) {
  for (auto &op : e.ops) {
    size_t k = 0;
    while (k < objs.size() && upper_case(objs[k].label) != upper_case(op.label)) k++;
    if (k == objs.size()) {
      set_error("transformation %s: no object labelled %s", e.tag.c_str(), op.label.c_str());
      return BG_ERR_ARG;
    }
    xf_compose(objs[k].xf, op.xf);
  }
  return BG_OK;
}

int parse_buffgeo(const char *path, std::vector<GeoObject> &objs) {
  std::vector<std::vector<std::string>> special;
  if (special_name(path, special)) {
    GeoObject o;
    o.label = special[0][1];
    xf_identity(o.xf);
    std::vector<int> lineno(special.size(), 0);
    MatDB none;
    int st = parse_object_lines(special, lineno, 0, path, ".", {}, none, o);
    if (st) return st;
    objs.push_back(o);
    return BG_OK;
  }
  FILE *f = std::fopen(path, "r");
  if (!f) { set_error("could not open %s", path); return BG_ERR_IO; }
  std::string dir = path;
  size_t slash = dir.find_last_of('/');
  dir = (slash == std::string::npos) ? std::string(".") : dir.substr(0, slash);
  std::vector<std::string> meshpath;
  std::string buf;
  int lineno = 0, start = 0;
  bool in = false;
  GeoObject cur;
  std::vector<std::vector<std::string>> body;
  std::vector<int> bodyline;
  MatDB db;
  bool inmat = false;
  std::string matname;
  std::vector<std::string> matlines;
  std::vector<int> matlineno;
  auto fail = [&](int ln, const char *msg) {
    std::fclose(f);
    set_error("%s:%d: %s", path, ln, msg);
    return BG_ERR_IO;
  };
  while (get_line(f, buf)) {
    lineno++;
    std::vector<std::string> tok = tokenize(buf.c_str());
    if (tok.empty() || tok[0][0] == '#') continue;
    if (inmat) {
      if (keyword_is(tok[0], "ENDMATERIAL")) {
        std::shared_ptr<const MatPropFn> fn;
        int st = matprop_parse_section(matname, matlines, matlineno, path, fn);
        if (st) { std::fclose(f); return st; }
        db.emplace_back(matname, fn);
        inmat = false;
      } else {
        matlines.push_back(buf);
        matlineno.push_back(lineno);
      }
      continue;
    }
    if (in) {
      if (keyword_is(tok[0], "ENDOBJECT")) {
        int st = parse_object_lines(body, bodyline, lineno, path, dir, meshpath, db, cur);
        if (st) { std::fclose(f); return st; }
        objs.push_back(cur);
        in = false;
      } else {
        body.push_back(tok);
        bodyline.push_back(lineno);
      }
    } else if (keyword_is(tok[0], "OBJECT")) {
      if (tok.size() != 2) return fail(lineno, "invalid OBJECT specification");
      cur = GeoObject{};
      cur.label = tok[1];
      xf_identity(cur.xf);
      body.clear();
      bodyline.clear();
      in = true;
      start = lineno;
    } else if (keyword_is(tok[0], "MESHPATH")) {
      if (tok.size() != 2) return fail(lineno, "invalid MESHPATH specification");
      meshpath.push_back(tok[1][0] == '/' ? tok[1] : dir + "/" + tok[1]);
    } else if (keyword_is(tok[0], "MATERIAL")) {
      // SWGGeometry.cc:318-330: one name, then the section up to ENDMATERIAL
      if (tok.size() == 1) return fail(lineno, "no name given for MATERIAL");
      if (tok.size() > 2) return fail(lineno, "syntax error");
      inmat = true;
      matname = tok[1];
      matlines.clear();
      matlineno.clear();
      start = lineno;
    } else {
      return fail(lineno, "syntax error");
    }
  }
  std::fclose(f);
  if (in) { set_error("%s:%d: OBJECT without ENDOBJECT", path, start); return BG_ERR_IO; }
  if (inmat) { set_error("%s:%d: MATERIAL without ENDMATERIAL", path, start); return BG_ERR_IO; }
  if (objs.empty()) { set_error("%s: no objects", path); return BG_ERR_IO; }
  return BG_OK;
}

}  // namespace bg
