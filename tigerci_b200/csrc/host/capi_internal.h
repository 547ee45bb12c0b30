// Shared helpers of the C ABI implementation (host and device parts).
#pragma once
#include <exception>
#include <string>

#include "../../../include/tigerci_sigma.h"
#include "plan.h"

namespace tci {
void set_error(const std::string& m);
int guard_status(const std::exception_ptr& ep);
void build_space_from_c(const tci_deck* d, CsfSpace& sp);
void operator_from_c(const tci_operator* op, const CsfSpace& sp, Operator& out);
// Device half of tci_sigma_init: a context from a host-built space and plan
// (chol: the host Cholesky vectors the plan was built for).
// refine (mixed form): finish every root as an FP64 Rayleigh quotient, 1 with a plain-FP64 sigma build
// (keeps the FP64 W), 2 with every term FP64 but the all-external one (default), 3 as 2 with the
// three-external contractions on the tensor cores too, 0 not at all.
// Local pair domains: the local space, its CSFs' indices in the non-local space of the same deck (the
// plan's layout), the heads of the pair-domain all-external term (7 int64 each, as tci_local_create takes
// them) with their domains, and the (aa|cc), (ac|ca) arrays of the all-external diagonal.
struct LocalSetup {
  CsfSpace loc;
  std::vector<long long> map;
  std::vector<int64_t> heads7, dom_idx;
  std::vector<int64_t> heads_lex;  // the lexical index of each heads7 entry's N-2 path
  std::vector<double> xdiag;
  // per N-2 head of the non-local plan (its dheads order): the slice of dh_dom holding the head's local
  // domain (sorted externals); length 0 for a head without local CSFs
  std::vector<int64_t> dh_off, dh_len;
  std::vector<int> dh_dom;
  // the N-1 heads of the non-local plan: CSF rows [s1_begin, s1_end) of each head (one row of n externals
  // per spin function) and the slice of s1_dom holding its local domain (length 0: no local CSFs)
  std::vector<int64_t> s1_begin, s1_end, s1_off, s1_len;
  std::vector<int> s1_dom;
};
void build_local_setup(const CsfSpace& loc, const CsfSpace& nl, const Operator& op, LocalSetup& ls);
// everything of build_local_setup but the all-external diagonal arrays (no operator needed)
void build_local_structure(const CsfSpace& loc, const CsfSpace& nl, LocalSetup& ls);
int ctx_from_plan(CsfSpace&& sp, Plan&& plan, const double* chol, int64_t device, int64_t precision, int64_t kblock,
                  tci_ctx** out, int64_t refine = 2, LocalSetup* ls = nullptr, tci_ctx* started = nullptr);
// A context started from the operator part of a plan (build_plan_operator_part): buffers of the integral banks
// allocated, the Cholesky vectors uploaded and the leading set-up steps run, so that the device builds the
// banks while the host builds the sigma tables; ctx_from_plan(..., started) completes it with the whole plan
// (and takes ownership of it, also on failure).
int ctx_begin_operator(const Plan& early, const double* chol, int64_t device, int64_t precision, int64_t kblock,
                       int64_t refine, tci_ctx** out);
// Uploads the plan's coupling-vector rows (plan.wv, n doubles) into a started context ahead of ctx_from_plan,
// which then skips them; throws on failure.
void ctx_upload_wv(tci_ctx* ctx, const double* wv, size_t n);
// Selects the GEMM steps that run on the tensor cores in the mixed form (tci_sigma_init_ex options[2]).
void ctx_set_tc_gemms(tci_ctx* ctx, int64_t mode);
// Device bytes of such a context: peak during set-up and held afterwards.
void ctx_device_bytes(const Plan& plan, int64_t precision, double* peak, double* resident, int64_t refine = 2);
}  // namespace tci
