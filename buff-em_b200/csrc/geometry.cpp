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
// is kept; the displacement is applied before the merge, as the one-time
// transformation is (:120-121).
static int read_gmsh(Object &o, const char *path, const double *disp) {
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
  if (disp)
    for (int i = 0; i < nv; i++)
      for (int k = 0; k < 3; k++) o.V[3 * i + k] += disp[k];
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

int load_object(Object &o, const char *meshfile, const double *disp) {
  o.meshfile = meshfile;
  int st = read_gmsh(o, meshfile, disp);
  if (st) return st;
  if (disp) for (int k = 0; k < 3; k++) o.origin[k] = disp[k];
  return init_faces(o);
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
      for (int j = 0; j < 4; j++) {
        for (int k = 0; k < 3; k++) {
          double s = 0.0;
          for (int i = 0; i < 4; i++) s += (i == j ? qb : qa) * o.V[3 * T[i] + k];
          tetP4.push_back(s);
        }
        tetP4.push_back(0.0);
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
  if (*end == 'i' || *end == 'j' || *end == 'I') { *re = 0; *im = a; return true; }
  if (*end == 0) { *re = a; *im = 0; return true; }
  const char *p = end;
  double b = std::strtod(p, &end);
  if (end == p || (*end != 'i' && *end != 'j' && *end != 'I')) return false;
  *re = a; *im = b;
  return true;
}

int parse_buffgeo(const char *path, std::vector<std::string> &meshes, std::vector<double> &disp,
                  std::vector<bg_material> &mats) {
  FILE *f = std::fopen(path, "r");
  if (!f) { set_error("cannot open geometry file %s", path); return BG_ERR_IO; }
  std::string dir = path;
  size_t slash = dir.find_last_of('/');
  dir = (slash == std::string::npos) ? std::string(".") : dir.substr(0, slash);
  const char *mp = std::getenv("BUFF_MESH_PATH");
  char line[1024];
  bool in = false;
  std::string mesh;
  double d[3] = {0, 0, 0};
  bg_material m{};
  int lineno = 0;
  while (std::fgets(line, sizeof line, f)) {
    lineno++;
    char *p = line;
    while (*p && std::isspace((unsigned char)*p)) p++;
    if (!*p || *p == '#') continue;
    char kw[64] = {0}, arg[512] = {0};
    int n = std::sscanf(p, "%63s %511[^\n]", kw, arg);
    std::string K = kw;
    for (auto &c : K) c = (char)std::toupper((unsigned char)c);
    if (K == "OBJECT") {
      in = true; mesh.clear(); d[0] = d[1] = d[2] = 0; m = bg_material{}; m.kind = BG_MAT_CONST_ISO;
      m.eps[0] = 1.0;
    } else if (K == "MESHFILE" && in && n == 2) {
      char fn[512];
      std::sscanf(arg, "%511s", fn);
      std::string cand = fn;
      if (fn[0] != '/') {
        cand = dir + "/" + fn;
        FILE *t = std::fopen(cand.c_str(), "r");
        if (!t && mp) cand = std::string(mp) + "/" + fn;
        if (t) std::fclose(t);
      }
      mesh = cand;
    } else if (K == "MATERIAL" && in && n == 2) {
      char nm[256];
      std::sscanf(arg, "%255s", nm);
      std::string M = nm;
      std::string U = M;
      for (auto &c : U) c = (char)std::toupper((unsigned char)c);
      if (U.rfind("CONST_EPS_", 0) == 0) {
        if (!parse_complex(M.c_str() + 10, &m.eps[0], &m.eps[1])) {
          std::fclose(f); set_error("%s:%d: bad permittivity %s", path, lineno, nm); return BG_ERR_IO; }
        m.kind = BG_MAT_CONST_ISO;
      } else if (U == "VACUUM") {
        m.kind = BG_MAT_CONST_ISO; m.eps[0] = 1.0; m.eps[1] = 0.0;
      } else {
        std::fclose(f); set_error("%s:%d: unsupported material %s (CONST_EPS_<value> only)", path, lineno, nm);
        return BG_ERR_IO;
      }
    } else if (K == "DISPLACED" && in) {
      if (std::sscanf(arg, "%lf %lf %lf", d, d + 1, d + 2) != 3) {
        std::fclose(f); set_error("%s:%d: bad DISPLACED", path, lineno); return BG_ERR_IO; }
    } else if (K == "ENDOBJECT" && in) {
      if (mesh.empty()) { std::fclose(f); set_error("%s:%d: object without MESHFILE", path, lineno); return BG_ERR_IO; }
      meshes.push_back(mesh); mats.push_back(m);
      disp.push_back(d[0]); disp.push_back(d[1]); disp.push_back(d[2]);
      in = false;
    } else if (K == "MATERIAL" || K == "MESHFILE") {
      std::fclose(f); set_error("%s:%d: %s outside OBJECT", path, lineno, kw); return BG_ERR_IO;
    } else {
      std::fclose(f); set_error("%s:%d: unsupported keyword %s", path, lineno, kw); return BG_ERR_IO;
    }
  }
  std::fclose(f);
  if (in) { set_error("%s: missing ENDOBJECT", path); return BG_ERR_IO; }
  if (meshes.empty()) { set_error("%s: no objects", path); return BG_ERR_IO; }
  return BG_OK;
}

}  // namespace bg
