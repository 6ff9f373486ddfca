// MPS checkpoints: a metadata file plus a raw block file.
//
// Mirrors qTensorTrain::save/load (mps/qtt.cpp:678-771) and the dense
// TensorTrain save/load (mps/tt.cpp, dtensor/dtensor.cpp:610-713): the raw
// file holds every block of every site tensor as dense column-major doubles,
// back to back in site order and block order, and the metadata records the
// MPS attributes (length, phy_dim, bond_dims, center, totalQ, phy_qn, id, the
// raw file name), each tensor's indices and each block's sector tuple and
// byte offset.  The reference writes its metadata with HDF5, which this
// build does not link; the metadata here is a versioned text file
// ("<fn>.ttmps") with the same fields, so a checkpoint moves between the two
// by translating the metadata only -- the raw block file has the same layout.
#pragma once

#include <string>

#include "dmrg_d.h"
#include "dmrg_q.h"

namespace ttb {

// wfn empty -> fn + "__T.bin"; the metadata goes to fn + ".ttmps".
void save(const qMPS& psi, const std::string& fn, const std::string& wfn = "");
// fn is the metadata file; data_prefix is prepended to the recorded raw file
// name (qTensorTrain::load(fn, dataPrefix)).
qMPS load_qmps(const std::string& fn, const std::string& data_prefix = "");

void save(const MPS& psi, const std::string& fn, const std::string& wfn = "");
MPS load_mps(const std::string& fn, const std::string& data_prefix = "");

}  // namespace ttb
