// Host-side data model of the MRSDCI sigma build (C++17, no CUDA types).
//
// The CSF space follows TigerCI's symmetric-group graphical approach (SGGA):
// a distinct-row table over spatial occupations (0/1/2 per orbital) whose
// paths through the internal orbitals are the "heads" of the CI vector, and
// Yamanouchi-Kotani spin functions enumerated by the SFT graph.
//   graph construction ........ tiger_fortran/graph_mod.f90:101-378
//   tree search / index vectors  tiger_fortran/graph_mod.f90:572-1589
//   spin functions ............. tiger_fortran/spin_mod.f90:99-522
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <map>
#include <stdexcept>

namespace tci {

using i64 = int64_t;

constexpr i64 kKillNumber = -1000000;   // tiger_fortran/global_var_mod.f90:72
constexpr i64 kFsnSize = 150;           // tiger_fortran/global_var_mod.f90:71
constexpr int kExcitationLevel = 2;     // tiger_fortran/graph_var_mod.f90:69

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Input deck fields that shape the CSF space (TigerCI keywords in brackets).
struct Deck {
  i64 num_orbitals = 0;    // NUMBER OF ORBITALS
  i64 num_frozen = 0;      // NUMBER OF FROZEN ORBITALS (subset of inactive)
  i64 num_inactive = 0;    // NUMBER OF INACTIVE ORBITALS
  i64 num_active = 0;      // NUMBER OF ACTIVE ORBITALS
  i64 num_elec = 0;        // NUMBER OF ELECTRONS
  i64 spin_mult = 1;       // SPIN MULTIPLICITY
  i64 num_ref = 0;         // NUMBER OF REFERENCES
  std::vector<int> refs;   // num_ref x num_internal occupations (row major)
  i64 num_internal() const { return num_inactive + num_active; }
  i64 num_external() const { return num_orbitals - num_internal(); }
};

// One internal path (head) at the internal/external border.
struct Head {
  i64 lex = 0;             // 1-based lexical index among paths ending at this vertex
  int kind = 0;            // 0 valence, 1 N-1, 2 N-2
  int singles = 0;         // internal open shells
  bool kept = false;       // survives excitation/frozen/spin/open-shell checks
  std::vector<int8_t> occ; // occupation of every internal orbital
  i64 domain = -1;         // index into CsfSpace::domains (N-1/N-2 only)
  // 0-based CSF offsets (reference's 1-based index vectors minus one)
  i64 off = -1;            // valence / N-1 block, or N-2 "ab" block
  i64 off_aa = -1;         // N-2 "aa" block
  int nsf = 0;             // spin functions of the block at `off`
  int nsf_aa = 0;          // spin functions of the "aa" block
};

struct CsfSpace {
  Deck deck;
  i64 n_int = 0, n_ext = 0;
  // graph (graph_mod.f90:101-378), levels 0..num_orbitals
  std::vector<i64> left_border, right_border, auxiliary;  // size num_orbitals+1
  std::vector<i64> y0, y1, y2;                            // 1-based vertices stored at [v]
  i64 num_vert = 0;
  i64 open_shells = 0;
  std::vector<i64> fsn;   // final spin-function counts (0 for disallowed counts)
  // heads per electron deficit: paths[0] valence, [1] N-1, [2] N-2; indexed by lex-1
  std::vector<Head> paths[3];
  // sorted external domains (0-based external indices), deduplicated like
  // allowed_virtuals_mod.f90:163-219
  std::vector<std::vector<int>> domains;
  i64 num_valence = 0, num_nm1 = 0, num_nm2 = 0, total_csfs = 0;
  i64 total_configurations = 0;  // abs(y0(num_vert))
  i64 removed = 0;
  // per-block statistics printed by index_vector_internal ("For n singles ...")
  std::map<int, i64> cfg_count[3];

  i64 vertex(i64 level, i64 elec) const { return auxiliary[level] + elec; }
  bool belong(i64 level, i64 elec) const;
};

// Optional per-path domains: for each N-1 / N-2 path (lex-1 order) the sorted
// list of allowed external indices (0-based); an empty outer vector means
// non-local (every path sees all externals).  A path may be given the list
// {-1} to mark it removed by the local criteria (num_allowed_virtuals = 0).
struct DomainSpec {
  std::vector<std::vector<int>> nm1, nm2;
};

void build_csf_space(const Deck& deck, const DomainSpec& dom, CsfSpace& out);

// ---------------------------------------------------------------------------
// Spin functions (spin_mod.f90).  Functions for s open shells are the first
// fsn(s) columns of the max-open-shell SFT ordering; open shell i (ascending
// orbital order) sits on arc i and arcs are coupled from the highest down.
struct SpinTables {
  int open_shells = 0;
  int spin_mult = 1;
  std::vector<i64> fsn_all;      // fsn before the final zeroing (graph_mod.f90:381-491)
  int nsf_max = 0;
  // spin_matrix(v, f): multiplicity at vertex v (0..open_shells) of function f
  std::vector<int> spin_matrix;  // (open_shells+1) x nsf_max, row major in v
  std::vector<int> sft;          // (open_shells-1) x nsf_max, row major in arc
  int mult(int v, int f) const { return spin_matrix[v * nsf_max + f]; }
};

void build_spin_tables(int open_shells, int spin_mult, SpinTables& out);

// Expansion of the fsn(s) spin functions for s open shells over spin strings
// (bit i set = beta on arc i+1), M_S = S.  coeff is nstr x nsf (row major).
struct SpinBasis {
  int s = 0, nsf = 0;
  std::vector<uint32_t> strings;
  std::vector<double> coeff;
  std::map<uint32_t, int> index;
};
const SpinBasis& spin_basis(const SpinTables& t, int s);

}  // namespace tci
