// C++ mirror of SPECFEM++'s kernel facade and forward time loop over libsfg's
// C ABI (include/sfg.h): what the reference's host driver keeps when its
// kernels move to libsfg.
//
//   domain_kernels       include/kokkos_kernels/domain_kernels.hpp:37-214
//                        (initialize, update_wavefields<medium>, compute_seismograms)
//   newmark              core/specfem/timescheme/newmark.tpp:10-128
//                        (predictor / corrector phases returning the degrees of
//                        freedom updated, seismogram sampling)
//   time_marching_forward core/specfem/solver/time_marching.tpp:8-131: the
//                        medium order of one step and the check that every
//                        degree of freedom and every element was updated
//
// Errors of the C ABI become std::runtime_error with the library's message,
// as the reference's kernels throw (program.cpp catches them).
#pragma once

#include <sstream>
#include <stdexcept>
#include <string>

#include "../../include/sfg.h"

namespace specfem_b200 {

enum class medium_tag : int { acoustic = SFG_MEDIUM_ACOUSTIC, elastic = SFG_MEDIUM_ELASTIC };

inline int checked(const sfg_handle *h, int rc) {
  if (rc < 0) {
    const char *m = sfg_last_error(h);
    throw std::runtime_error(std::string("libsfg error ") + std::to_string(rc) + ": " + (m ? m : ""));
  }
  return rc;
}

// The kernels of one 2D forward simulation on a libsfg handle.
class domain_kernels {
 public:
  explicit domain_kernels(sfg_handle *h) : h_(h) {}
  // compute_mass_matrix + invert_mass_matrix (the handle was created with dt)
  void initialize() { checked(h_, sfg_initialize(h_)); }
  template <medium_tag M>
  int update_wavefields(int istep) {
    return checked(h_, sfg_update_wavefields(h_, static_cast<int>(M), istep));
  }
  void compute_seismograms(int isig_step) { checked(h_, sfg_compute_seismograms(h_, isig_step)); }
  sfg_handle *handle() const { return h_; }

 private:
  sfg_handle *h_;
};

// Newmark time scheme of a forward simulation.
class newmark {
 public:
  newmark(sfg_handle *h, int nstep, int nstep_between_samples)
      : h_(h), nstep_(nstep), nsb_(nstep_between_samples > 0 ? nstep_between_samples : 1) {}
  int apply_predictor_phase_forward(medium_tag m) { return checked(h_, sfg_predictor(h_, static_cast<int>(m))); }
  int apply_corrector_phase_forward(medium_tag m) { return checked(h_, sfg_corrector(h_, static_cast<int>(m))); }
  bool compute_seismogram(int istep) const { return istep % nsb_ == 0; }
  int get_seismogram_step() const { return isig_; }
  void increment_seismogram_step() { ++isig_; }
  int get_max_timestep() const { return nstep_; }

 private:
  sfg_handle *h_;
  int nstep_, nsb_;
  int isig_ = 0;
};

// time_marching<forward, dim2, 5>::run: per step the predictor of every
// medium, then update_wavefields and the corrector of the acoustic medium,
// then of the elastic medium, then the seismograms; after every step the
// counts of degrees of freedom and elements updated are checked.
inline void time_marching_forward(domain_kernels &kernels, newmark &ts) {
  constexpr auto acoustic = medium_tag::acoustic;
  constexpr auto elastic = medium_tag::elastic;
  kernels.initialize();
  sfg_info info;
  checked(kernels.handle(), sfg_get_info(kernels.handle(), &info));
  const int total_dof_to_be_updated =
      2 * (info.nglob_elastic * info.ncomp_elastic + info.nglob_acoustic);
  const int total_elements_to_be_updated = info.nspec;
  const int nstep = ts.get_max_timestep();
  for (int istep = 0; istep < nstep; ++istep) {
    int dofs_updated = 0;
    int elements_updated = 0;
    dofs_updated += ts.apply_predictor_phase_forward(acoustic);
    dofs_updated += ts.apply_predictor_phase_forward(elastic);
    elements_updated += kernels.update_wavefields<acoustic>(istep);
    dofs_updated += ts.apply_corrector_phase_forward(acoustic);
    elements_updated += kernels.update_wavefields<elastic>(istep);
    dofs_updated += ts.apply_corrector_phase_forward(elastic);
    if (ts.compute_seismogram(istep)) {
      kernels.compute_seismograms(ts.get_seismogram_step());
      ts.increment_seismogram_step();
    }
    if (dofs_updated != total_dof_to_be_updated) {
      std::ostringstream message;
      message << "The time loop has not updated all the degrees of freedom. Only " << dofs_updated
              << " out of " << total_dof_to_be_updated << " degrees of freedom have been updated.";
      throw std::runtime_error(message.str());
    }
    if (elements_updated != total_elements_to_be_updated) {
      std::ostringstream message;
      message << "The time loop has not updated all the elements. Only " << elements_updated << " out of "
              << total_elements_to_be_updated << " elements have been updated.";
      throw std::runtime_error(message.str());
    }
  }
  checked(kernels.handle(), sfg_synchronize(kernels.handle()));
}

}  // namespace specfem_b200
