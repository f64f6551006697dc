// specfem2d_facade: a forward simulation driven through the C++ facade
// (specfem_facade.hpp), the reference's time loop over libsfg.
//
//   specfem2d_facade DATABASE SETUP OUT
//
// DATABASE  a SPECFEM2D database.bin;
// SETUP     text: "dt nstep nstep_between_samples elastic_wave(0 P-SV, 1 SH)",
//           then "nsrc" and one line per force source
//           "x z f0 factor tshift angle stf(SFG_STF_*)", then "nrec ntypes type..."
//           and one line per receiver "x z";
// OUT       raw float32 seismograms [nsig][ntypes][nrec][2].
// Prints the degrees of freedom and elements checked per step.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "specfem_facade.hpp"

int main(int argc, char **argv) {
  if (argc != 4) {
    std::cerr << "usage: specfem2d_facade DATABASE SETUP OUT\n";
    return 2;
  }
  try {
    std::ifstream in(argv[2]);
    double dt;
    int nstep, nsb, wave, nsrc;
    in >> dt >> nstep >> nsb >> wave >> nsrc;
    std::vector<sfg_source2d> src(nsrc);
    for (auto &s : src) {
      s = sfg_source2d{};
      in >> s.x >> s.z >> s.f0 >> s.factor >> s.tshift >> s.angle >> s.stf;
      s.kind = SFG_SOURCE_FORCE;
    }
    int nrec, ntypes;
    in >> nrec >> ntypes;
    std::vector<int> types(ntypes);
    for (int &t : types) in >> t;
    std::vector<double> rx(nrec), rz(nrec);
    for (int r = 0; r < nrec; ++r) in >> rx[r] >> rz[r];
    if (!in) throw std::runtime_error("malformed setup file");

    sfg_options opt{};
    opt.dt = dt;
    opt.nstep = nstep;
    opt.nshots = 1;
    opt.nstep_between_samples = nsb;
    sfg_handle *h = nullptr;
    if (sfg_create2d_from_database(argv[1], wave, &opt, &h) != SFG_OK) throw std::runtime_error(sfg_last_error(nullptr));
    specfem_b200::checked(h, sfg_set_sources(h, nsrc, src.data()));
    specfem_b200::checked(h, sfg_set_receivers(h, nrec, rx.data(), rz.data(), 0.0, ntypes, types.data()));

    specfem_b200::domain_kernels kernels(h);
    specfem_b200::newmark ts(h, nstep, nsb);
    specfem_b200::time_marching_forward(kernels, ts);

    sfg_info info;
    sfg_get_info(h, &info);
    const size_t n = size_t(info.nsig) * info.ntypes * info.nrec * 2;
    std::vector<float> seis(n);
    specfem_b200::checked(h, sfg_get_seismograms(h, seis.data(), n));
    std::ofstream out(argv[3], std::ios::binary);
    out.write(reinterpret_cast<const char *>(seis.data()), std::streamsize(n * sizeof(float)));
    std::printf("steps %d, elements %d, degrees of freedom %d per phase pair, samples %d\n", nstep, info.nspec,
                info.nglob_elastic * info.ncomp_elastic + info.nglob_acoustic, info.nsig);
    sfg_destroy(h);
  } catch (const std::exception &e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
