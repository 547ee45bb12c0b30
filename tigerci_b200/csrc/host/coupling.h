// Coupling-coefficient engine: matrix elements of spin-free one- and
// two-electron operators between the SGGA spin functions of two spatial
// configurations, evaluated through the spin-string expansion of each CSF.
//
// CSF convention (fixes every relative sign):
//   |m,k> = sum_x Theta_k(x) a+_{q_s x_s} ... a+_{q_1 x_1} prod_{d asc} a+_{d,alpha} a+_{d,beta} |0>
// with open shells q_1 < ... < q_s on arcs 1..s and Theta the genealogical
// (Yamanouchi-Kotani) coefficients of spin.cpp.  With this ordering a singlet
// external pair |ab> and the doubly occupied |aa> satisfy the SCEP relation
// used by tiger_fortran/scepmaker_mod.f90:121-165 (symmetric matrix with
// sqrt(2)*C_aa on the diagonal).
#pragma once
#include "tci_host.h"

#include <memory>
#include <mutex>

namespace tci {

using Det = unsigned __int128;

struct Config {
  std::vector<int8_t> occ;  // per orbital 0/1/2
};

struct CsfExpansion {
  int s = 0, nsf = 0;
  std::vector<int> open;             // open-shell orbitals, ascending
  std::vector<Det> dets;             // canonical determinant per spin string
  double sign = 1.0;                 // (-1)^{s(s-1)/2}
  const SpinBasis* basis = nullptr;  // Theta (nstr x nsf)
  std::map<Det, int> index;          // det -> string row
};

// Spin-summed operator: E_pq (r = s = -1) or e_pq,rs = sum a+_p a+_r a_s a_q.
struct Op {
  int p, q, r = -1, s = -1;
};

class CouplingEngine {
 public:
  explicit CouplingEngine(const SpinTables& t) : tables_(t) {}
  const CsfExpansion& expand(const Config& c);
  // out is nsf(L) x nsf(R), row major, overwritten.
  void matrix(const Config& L, const Config& R, const Op& op, std::vector<double>& out);
  // Accumulate coef * <L|op|R> into out (nsf(L) x nsf(R)).
  void accumulate(const Config& L, const Config& R, const Op& op, double coef, std::vector<double>& out);
  // The same for configurations already expanded (by this or another engine).
  void matrix(const CsfExpansion& L, const CsfExpansion& R, const Op& op, std::vector<double>& out);
  void accumulate(const CsfExpansion& L, const CsfExpansion& R, const Op& op, double coef, std::vector<double>& out);
  const SpinTables& tables() const { return tables_; }

 private:
  const SpinTables& tables_;
  std::mutex mu_;  // expand() may be called from several threads; cached entries never move
  std::map<std::vector<int8_t>, std::unique_ptr<CsfExpansion>> cache_;
};

}  // namespace tci
