// Overlaps, expectation values and Sz correlators of MPS on the device.
//
// psiphi / psiHphi follow mps/observables.cpp:26-103 (psiHphi) and :383-450
// (psiphi) for qMPS and dense MPS: a left-to-right chain of block
// contractions closed by boundary tensors of ones.  measure_sz is a
// build-side observable (the reference has none): <Sz_i> and <Sz_i Sz_j> from
// left/right transfer environments, with Sz applied as a diagonal scale of
// the physical mode, normalised by <psi|psi>.
#pragma once

#include <vector>

#include "dmrg_d.h"
#include "dmrg_q.h"

namespace ttb {

double psiphi(const qMPS& psi, const qMPS& phi);
double psiHphi(const qMPS& psi, const qMPO& H, const qMPS& phi);
// sz: L entries; szsz: L*L row-major, symmetric, diagonal <Sz_i^2> = 1/4.
void measure_sz(const qMPS& psi, std::vector<double>& sz, std::vector<double>& szsz);

double psiphi(const MPS& psi, const MPS& phi);
double psiHphi(const MPS& psi, const MPO& H, const MPS& phi);
void measure_sz(const MPS& psi, std::vector<double>& sz, std::vector<double>& szsz);

}  // namespace ttb
