// buff-scatter-style driver on the libbuff-compatible C++ layer
// (pattern of buff-scatter.cc:236-347 and unit-test-LFField.cc:50-71).
// usage: scatter_driver <geo.buffgeo> <omega> [geometry-only | extras]
//   extras: also the full PFT columns, the fields at one point and the
//   buff-neq flux of the geometry
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../buff-em_b200/compat/libbuff_b200.hpp"

using namespace buff_b200;

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  try {
    SWGGeometry G(argv[1]);
    std::printf("objects %d bfs %d\n", G.NumObjects, G.TotalBFs);
    const SWGVolume *O = G.Objects[G.NumObjects - 1].get();
    int no = -2;
    std::printf("label %s %d\n", O->Label.c_str(), G.GetObjectByLabel(O->Label.c_str(), &no) == O ? no : -1);
    cdouble eps = G.GetEps(G.NumObjects - 1, cdouble(std::atof(argv[2]), 0.0));
    std::printf("eps %.17g %.17g\n", eps.real(), eps.imag());
    const double X0[3] = {0.1, 0.2, 0.3};
    cdouble Q[3][3];
    G.GetEpsTensor(G.NumObjects - 1, cdouble(std::atof(argv[2]), 0.0), X0, Q);
    std::printf("qzz %.17g %.17g\n", Q[2][2].real(), Q[2][2].imag());
    std::printf("last %d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", O->NumVertices, O->NumInteriorFaces,
                O->Origin[0], O->Origin[1], O->Origin[2], O->Vertices[0], O->Vertices[1], O->Vertices[2]);
    if (argc > 3 && !std::strcmp(argv[3], "geometry-only")) return 0;
    cdouble Omega(std::atof(argv[2]), 0.0);
    HMatrix *M = G.AllocateVIEMatrix();
    HVector *J = G.AllocateRHSVector();
    G.AssembleVIEMatrix(Omega, M);
    M->LUFactorize();
    const cdouble E0[3] = {1.0, 0.0, 0.0};
    const double nHat[3] = {0.0, 0.0, 1.0};
    PlaneWave PW(E0, nHat);
    G.AssembleRHSVector(Omega, &PW, J);
    M->LUSolve(J);
    std::vector<double> P = G.GetPFTMatrix(J, Omega, &PW);
    std::printf("J0 %.17g %.17g\n", J->GetEntry(0).real(), J->GetEntry(0).imag());
    std::printf("PAbs %.17g PScat %.17g\n", P[0], P[1]);
    if (argc > 3 && !std::strcmp(argv[3], "extras")) {
      std::vector<double> P8 = G.GetPFTMatrixFull(J, Omega, &PW);
      std::printf("Fz %.17g\n", P8[4]);
      const double X[3] = {0.3, -0.2, 2.5};
      cdouble EH[6];
      G.GetFields(&PW, J, Omega, X, EH);
      std::printf("Ex %.17g %.17g\n", EH[0].real(), EH[0].imag());
      std::printf("Hy %.17g %.17g\n", EH[4].real(), EH[4].imag());
      BNEQ NEQ(G);
      std::vector<double> F = NEQ.GetFlux(Omega);
      std::printf("PRad %.17g\n", F[1]);
    }
    delete M;
    delete J;
  } catch (const Error &e) {
    std::fprintf(stderr, "error %d: %s\n", e.status, e.what());
    return 1;
  }
  return 0;
}
