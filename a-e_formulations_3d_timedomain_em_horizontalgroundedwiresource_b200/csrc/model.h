// Model description and readers for the reference's direct-mode input files.
//
// Mirrors the inputs CalcNonstat3DLine reads (CalcNonstat3DLine/vec_prep_data.cpp:83-257,
// time_approx.cpp:243-287 inputvec, vec_prep_data.cpp:834-853 Read_infite0,
// TaskSP.cpp:467-597, give_out_vec_loop.cpp:44-73, vec_prep_data.cpp:982-1270
// LoadAndInitCurrent).  All indices are converted to 0-based on load.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace tdem {

constexpr double kMu0 = 4.0e-7 * 3.14159265358979;  // MU_0 of vfem_const.h

struct Dipole {
  int elem = -1;                 // element holding the dipole
  double ksi = 0, eta = 0, zeta = 0;  // local coordinates in [0,1]
  double dx = 0, dy = 0, dz = 0;      // dipole vector (wire length / nSrsRazb)
};

struct Model {
  // mesh
  int n_nodes = 0, n_elem = 0, n_bound_nodes = 0, n_edges = 0;
  std::vector<std::array<double, 3>> xyz;
  std::vector<std::array<int, 8>> nver;       // element nodes
  std::vector<int> nvkat;                     // element material (0-based)
  std::vector<int> l13d;                      // boundary nodes
  std::vector<std::array<int, 12>> ed;        // element edges
  std::vector<std::array<int, 2>> edge_nodes; // edge end nodes (lower, upper)
  // materials (per material index)
  std::vector<double> sigma, sigma0, mu;      // mu in H/m
  // time grid
  std::vector<double> time;
  std::vector<double> currentfunction;        // empty when no source file is needed
  double print_left = 0, print_right = 0;
  // sources and receivers
  int npls = 0;
  std::vector<std::array<double, 6>> wires;   // A(x,y,z), B(x,y,z) per source
  int n_srs_razb = 500;
  std::vector<std::vector<Dipole>> dipoles;   // per source
  std::vector<std::array<double, 3>> rec_b, rec_e;
  std::vector<int> rec_b_ig, rec_e_ig;        // per-source receiver ranges (npls+1)
  int n_neib = 5;
  bool fdirect = false;
  double eps_reg = 1e-12;
  // primary-secondary mode (fdirect 0): the edges whose normal field enters the
  // source (mtrsizeforE0, one flag per edge) and the name in the normal-field files
  // m<pname>.enor.NNNN (PName)
  std::vector<char> edge_anom;
  int n_anom = 0;
  std::string pname;
  int anomal_type = 0;  // AnomalType: nonzero when each anomaly has its own normal-field files
  int anomaly = -1;     // ia: the anomaly of this run (file suffix _<ia>)
  // derived
  std::vector<char> edge_bound;               // Dirichlet edge flag
  std::string dir;
};

// Reads every input of one working directory.  Returns "" or an error message.
std::string load_model(const std::string& dir, Model& m);

// Initial field on the edges (n_edges x npls, column-major): a0.edge / e0.edge
// when present, else the nodal a0.dat (A-form) / v3a.dat (E-form) projected onto
// the edges (CalcNonstat3DLine time_approx.cpp:816-889, E-form time_approx.cpp:856-901).
std::string load_initial_field(const Model& m, bool eform, std::vector<double>& u0);
// The same for the npls sources whose files are in dir, on the mesh of m.
std::string load_initial_field(const Model& m, const std::string& dir, int npls, bool eform,
                               std::vector<double>& u0);

// Several direct-mode models that differ only in their sources and receivers (the
// same mesh, materials, time grid, current function and printed range) as one model
// with all their sources, in order, each with its own receivers (the per-source
// receiver ranges rec_*_ig index the concatenated receiver lists).  The result keeps
// parts[0].dir.  Returns "" or why the parts cannot be merged.
std::string merge_models(const std::vector<Model>& parts, Model& out);

// Full symmetric CSR pattern over all edges (both triangles, sorted columns).
void edge_pattern(const Model& m, std::vector<int64_t>& rowptr, std::vector<int>& col);

// Dipole locations: each wire split into n_srs_razb dipoles placed in the first
// element (in file order) whose box (+-1e-3) holds them with local coordinates in
// (-0.01, 1.01), as LoadAndInitCurrent does (vec_prep_data.cpp:1050-1183).
std::string locate_dipoles(Model& m);

// Greedy element colouring for assembly without atomics: elements in file order take
// the lowest colour (< 64) that no element sharing an edge holds yet.  `order` lists
// the elements colour by colour (ascending inside a colour), colour c in
// [cstart[c], cstart[c + 1]).  Returns "" or an error when 64 colours do not suffice.
std::string element_colouring(const Model& m, std::vector<int>& order, std::vector<int>& cstart);

// Primary-secondary mode: the normal field of the anomalous edges (m.edge_anom) as
// edge values, in the reference's scaling f * len / 2.
struct NormalField {
  std::vector<int> idx;      // anomalous edges, ascending
  std::vector<double> len;   // their lengths
  std::vector<double> e0;    // E-form: layer 0 on every edge and source (-grad V of v3n.dat)
};

// Builds the anomalous-edge list; for the E-formulation also layer 0 from the normal
// potential v3n.dat (E2/time_approx.cpp:1384-1412).
std::string init_normal_field(const Model& m, bool eform, NormalField& nf);

// File of layer `layer` of the normal field: <dir>/m<PName>.enor.NNNN, with the suffix
// _<ia> when AnomalType is set (time_approx.cpp:1280-1287).
std::string normal_field_file(const Model& m, int layer);

// Layer `layer` of the normal field on every edge and source (n_edges x npls,
// source-major): layer 0 of the E-formulation from nf.e0, otherwise the float32 file
// m<PName>.enor.NNNN on the anomalous edges and 0 elsewhere (time_approx.cpp:1263-1348).
std::string normal_field_layer(const Model& m, const NormalField& nf, int layer, std::vector<double>& out);

// The E-formulation's source values of the step to layer `it` with history layers t1
// (and t2): minus the time derivative of the normal field, two-point, or three-point
// when `three_point` (E2/time_approx.cpp:1419-1431, E3/time_approx.cpp:1400-1460).
std::string normal_field_rate(const Model& m, const NormalField& nf, int it, int t1, int t2, bool three_point,
                              std::vector<double>& out);

}  // namespace tdem
