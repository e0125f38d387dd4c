// The reference's on-disk cache of frequency-independent near-field
// integrals (FIBBICache::Store / PreLoad, FIBBICache.cc:272-463), read and
// written from the device-resident near table.
//
// File layout (native endianness, as the reference writes it): the 13 bytes
// "FIBBI_GCACHE\0", then records of 27 floats (search key) followed by 6
// doubles (the static integrals F0..F5 that GetGMatrixElement combines as
// (F0 - F1/k^2) + ik (F2 - F3/k^2) + (ik)^2 (F4 - F5/k^2)).  The key of a
// basis-function pair (a, b) of one object is the float differences
// QM_a, V1_a, V2_a, V3_a, QP_b, QM_b, V1_b, V2_b, V3_b minus QP_a
// (GetFIBBICacheKey, FIBBICache.cc:133-160).  Lookups compare the key bits
// exactly, as the reference's map does: a displaced copy of an object finds
// only the records whose float differences the displacement leaves unchanged
// (about two thirds on the synthetic spheres).  The reference stores the
// pairs with nf_b >= nf_a of one object, which are exactly the near pairs here.
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.h"

namespace bg {

static const char kFibbiSig[] = "FIBBI_GCACHE";   // written with its terminating NUL: 13 bytes
static const size_t kSigBytes = sizeof(kFibbiSig);
static const size_t kKeyFloats = 27, kDataDoubles = 6;
static const size_t kRecBytes = kKeyFloats * sizeof(float) + kDataDoubles * sizeof(double);

static void pair_key(const Object &o, int fa, int fb, float *K) {
  const Face &A = o.F[fa], &B = o.F[fb];
  const double *QPA = o.V.data() + 3 * A.iQP;
  const int idx[9] = {A.iQM, A.iV1, A.iV2, A.iV3, B.iQP, B.iQM, B.iV1, B.iV2, B.iV3};
  for (int r = 0; r < 9; r++) {
    const double *X = o.V.data() + 3 * idx[r];
    for (int c = 0; c < 3; c++) K[3 * r + c] = (float)(X[c] - QPA[c]);
  }
}

// all near pairs (global indices, a <= b) and their table rows, on the host
static int near_table(bg_geometry *g, std::vector<int2> &pairs, std::vector<double> &data) {
  NearData &nd = g->near;
  pairs.resize(nd.npairs);
  data.resize((size_t)nd.npairs * kDataDoubles);
  if (nd.npairs) {
    BG_CUDA_TRY(cudaMemcpy(pairs.data(), nd.pairs, sizeof(int2) * nd.npairs, cudaMemcpyDeviceToHost));
    BG_CUDA_TRY(cudaMemcpy(data.data(), nd.fibbi, sizeof(double) * kDataDoubles * nd.npairs, cudaMemcpyDeviceToHost));
  }
  return BG_OK;
}

}  // namespace bg

using namespace bg;

extern "C" {

int bg_fibbi_store(bg_geometry *g, int obj, const char *path, int *written) {
  if (!g || !path || obj < 0 || obj >= (int)g->objs.size()) {
    set_error("bg_fibbi_store: bad arguments");
    return BG_ERR_ARG;
  }
  int st = bg_geometry_precompute(g);
  if (st) return st;
  std::vector<int2> pairs;
  std::vector<double> data;
  if ((st = near_table(g, pairs, data))) return st;
  FILE *f = std::fopen(path, "wb");
  if (!f) { set_error("bg_fibbi_store: cannot open %s", path); return BG_ERR_IO; }
  bool ok = std::fwrite(kFibbiSig, kSigBytes, 1, f) == 1;
  const Object &o = g->objs[obj];
  int lo = g->bfOffset[obj], hi = g->bfOffset[obj + 1], n = 0;
  float key[kKeyFloats];
  for (size_t k = 0; ok && k < pairs.size(); k++) {
    int a = pairs[k].x, b = pairs[k].y;
    if (a < lo || a >= hi) continue;
    pair_key(o, a - lo, b - lo, key);
    ok = std::fwrite(key, sizeof key, 1, f) == 1 &&
         std::fwrite(data.data() + kDataDoubles * k, sizeof(double) * kDataDoubles, 1, f) == 1;
    n++;
  }
  if (std::fclose(f) != 0) ok = false;
  if (!ok) { set_error("bg_fibbi_store: write to %s failed", path); return BG_ERR_IO; }
  if (written) *written = n;
  return BG_OK;
}

int bg_fibbi_load(bg_geometry *g, int obj, const char *path, int *matched) {
  if (!g || !path || obj < 0 || obj >= (int)g->objs.size()) {
    set_error("bg_fibbi_load: bad arguments");
    return BG_ERR_ARG;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) { set_error("bg_fibbi_load: cannot open %s", path); return BG_ERR_IO; }
  std::fseek(f, 0, SEEK_END);
  long size = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  char sig[sizeof(kFibbiSig)];
  if (size < (long)kSigBytes || std::fread(sig, kSigBytes, 1, f) != 1 || std::memcmp(sig, kFibbiSig, kSigBytes) != 0) {
    std::fclose(f);
    set_error("bg_fibbi_load: %s is not a FIBBI cache file", path);
    return BG_ERR_IO;
  }
  if ((size - (long)kSigBytes) % (long)kRecBytes != 0) {
    std::fclose(f);
    set_error("bg_fibbi_load: %s has a size that is not a whole number of records", path);
    return BG_ERR_IO;
  }
  long nrec = (size - (long)kSigBytes) / (long)kRecBytes;
  std::unordered_map<std::string, std::vector<double>> table;
  table.reserve((size_t)nrec * 2);
  std::vector<char> rec(kRecBytes);
  for (long r = 0; r < nrec; r++) {
    if (std::fread(rec.data(), kRecBytes, 1, f) != 1) {
      std::fclose(f);
      set_error("bg_fibbi_load: %s: short read at record %ld", path, r);
      return BG_ERR_IO;
    }
    std::vector<double> d(kDataDoubles);
    std::memcpy(d.data(), rec.data() + kKeyFloats * sizeof(float), sizeof(double) * kDataDoubles);
    table.emplace(std::string(rec.data(), kKeyFloats * sizeof(float)), std::move(d));
  }
  std::fclose(f);
  int st = bg_geometry_precompute(g);
  if (st) return st;
  std::vector<int2> pairs;
  std::vector<double> data;
  if ((st = near_table(g, pairs, data))) return st;
  const Object &o = g->objs[obj];
  int lo = g->bfOffset[obj], hi = g->bfOffset[obj + 1], n = 0;
  float key[kKeyFloats];
  for (size_t k = 0; k < pairs.size(); k++) {
    int a = pairs[k].x, b = pairs[k].y;
    if (a < lo || a >= hi) continue;
    pair_key(o, a - lo, b - lo, key);
    auto it = table.find(std::string(reinterpret_cast<const char *>(key), sizeof key));
    if (it == table.end()) continue;
    std::memcpy(data.data() + kDataDoubles * k, it->second.data(), sizeof(double) * kDataDoubles);
    n++;
  }
  if (n && g->near.npairs)
    BG_CUDA_TRY(cudaMemcpy(g->near.fibbi, data.data(), sizeof(double) * kDataDoubles * g->near.npairs,
                           cudaMemcpyHostToDevice));
  if (matched) *matched = n;
  return BG_OK;
}

}  // extern "C"
