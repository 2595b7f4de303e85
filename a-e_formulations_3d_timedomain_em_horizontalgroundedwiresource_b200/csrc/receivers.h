// Receiver operators: the value of a field component at a receiver is a fixed
// linear functional of the edge solution, precomputed once per model.
//
// The reference evaluates receivers by a local L2 smoothing
// (CalcNonstat3DLine/OutputResultant3d.cpp:343-515, Subdomain.cpp:142-441):
// element-centre values of the field (A or E: T_Brick::Calc_value_inside_hex;
// curl: Calc_rotor_inside_hex) weighted by the row sums of the nodal mass matrix
// form the right-hand side of a nodal mass-matrix system on a neighbourhood of
// the receivers' elements (n_neib levels, per material for E-type values), and
// the receiver value is the trilinear interpolation of that nodal solution.
// Because every stage is linear, value = w^T u with a sparse row w over edges:
// w is obtained here by one solve with the (symmetric) mass matrix per receiver
// instead of one solve per time layer.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "model.h"

namespace tdem {

struct ReceiverOperator {
  int nrec = 0;                  // receivers
  int ncomp = 3;                 // components per receiver
  std::vector<int64_t> rowptr;   // rows = comp * nrec + receiver
  std::vector<int> col;          // edge ids
  std::vector<double> val;
  std::vector<int> src;          // source whose field each row samples
  std::vector<int> elem;         // element holding each receiver
};

// curl = false: field value (A or E) at the element centres, one subdomain per
// material; curl = true: curl of the field, one subdomain over all materials.
// owner[i] is the source index whose solution receiver i samples.
std::string build_receiver_operator(const Model& m, const std::vector<std::array<double, 3>>& pts,
                                    const std::vector<int>& owner, bool curl, ReceiverOperator& out);

}  // namespace tdem
