// TorchScript-visible operators over the C ABI (torch.ops.admp_b200.*), with
// C++ autograd, so that CoulombForceModule, GaussianDampingForceModule,
// SiteForceModule and QEqForceModule can be compiled with torch.jit.script
// and saved as the reference's modules can (test_jit.py).  Every energy call
// produces the gradients the backward needs in the same launch sequence, as
// the Python autograd functions of admp_b200.ops do.
//
//   coulomb_pbc(pos, box, pairs, ds, bs, q, kappa, kmesh, spacing, ethresh,
//               ke, rspace, kspace, slab, axis) -> [E, comps, kmesh]
//                 pme.py:261-310 (real, reciprocal, self, non-neutral, slab)
//   coulomb_obc(pairs, ds, bs, q, ke) -> E                     pme.py:529-561
//   damping(ds, q, eta, pairs, bs, ke) -> E                    qeq.py:60-129
//   site(q, chi, hardness) -> E                                qeq.py:159-209
//
// Inputs are in the standardised (nframes, ...) layout of BaseForceModule.
#include <ATen/cuda/CUDAContext.h>
#include <torch/library.h>
#include <torch/torch.h>

#include <cmath>
#include <vector>

#include "admp_b200.h"

namespace {

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

// Status -> the exception types of the Python layer (admp_b200._lib.check):
// bad arguments / mesh -> ValueError, bad index -> IndexError, else RuntimeError.
void check(int st, const char* what) {
  if (st == ADMP_OK) return;
  TORCH_CHECK_VALUE(st != ADMP_ERR_BAD_ARG && st != ADMP_ERR_MESH, what, ": ", admp_last_error_message());
  TORCH_CHECK_INDEX(st != ADMP_ERR_BAD_INDEX, what, ": ", admp_last_error_message());
  TORCH_CHECK(false, what, ": ", admp_last_error_message(), " [", admp_status_string(st), "]");
}

int dtype_code(const Tensor& t) {
  TORCH_CHECK(t.scalar_type() == torch::kDouble || t.scalar_type() == torch::kFloat,
              "admp_b200 ops take float64 or float32 tensors");
  return t.scalar_type() == torch::kDouble ? ADMP_F64 : ADMP_F32;
}

void* stream_of(const Tensor& t) {
  TORCH_CHECK(t.is_cuda(), "admp_b200 ops run on CUDA tensors (there is no CPU path)");
  return (void*)at::cuda::getCurrentCUDAStream(t.device().index()).stream();
}

template <typename X>
X* ptr(const Tensor& t) {
  return t.defined() ? (X*)t.data_ptr() : nullptr;
}

Tensor f64(int64_t n, const Tensor& like) {
  return torch::zeros({n}, like.options().dtype(torch::kDouble));
}

// Mesh per frame: explicit kmesh, ceil(L / spacing) or ceil(2 kappa L / (3 ethresh^0.2))
// (pme.py:380-392), with the same double arithmetic as the Python modules.
std::vector<int> kmesh_per_frame(const Tensor& box, double kappa, const std::vector<int64_t>& kmesh,
                                 const std::vector<double>& spacing, double ethresh) {
  const int64_t nf = box.size(0);
  std::vector<int> km(3 * nf);
  Tensor diag;
  if (kmesh.empty()) diag = torch::diagonal(box.detach(), 0, 1, 2).to(torch::kCPU, torch::kDouble).contiguous();
  for (int64_t f = 0; f < nf; ++f)
    for (int d = 0; d < 3; ++d) {
      if (!kmesh.empty()) {
        km[3 * f + d] = (int)kmesh[d];
      } else {
        const double L = diag.data_ptr<double>()[3 * f + d];
        km[3 * f + d] = spacing.empty() ? (int)std::ceil(2 * kappa * L / (3.0 * std::pow(ethresh, 1.0 / 5.0)))
                                        : (int)std::ceil(L / spacing[d]);
      }
    }
  return km;
}

class CoulombPBC : public torch::autograd::Function<CoulombPBC> {
 public:
  static variable_list forward(AutogradContext* ctx, Tensor pos, Tensor box, Tensor ds, Tensor q, Tensor pairs,
                               Tensor bs, double kappa, std::vector<int64_t> kmesh, std::vector<double> spacing,
                               double ethresh, double ke, bool rspace, bool kspace, bool slab, int64_t axis) {
    const int dt = dtype_code(pos);
    void* st = stream_of(pos);
    const int64_t nf = pos.size(0), N = pos.size(1), P = pairs.size(1);
    const bool need = pos.requires_grad() || box.requires_grad() || ds.requires_grad() || q.requires_grad();
    Tensor E_real = f64(nf, pos), E_recip = f64(nf, pos);
    Tensor terms = torch::zeros({nf, 5}, pos.options().dtype(torch::kDouble));
    Tensor gpos, gbox, gds, gq;
    if (need) {
      gpos = torch::zeros_like(pos);
      gbox = torch::zeros_like(box);
      gds = torch::zeros_like(ds);
      gq = torch::zeros_like(q);
    }
    std::vector<int> km = kspace ? kmesh_per_frame(box, kappa, kmesh, spacing, ethresh)
                                 : std::vector<int>(3 * nf, 1);
    if (rspace && P > 0)
      check(admp_pair_energy(dt, ADMP_PAIR_EWALD, (int)nf, (int)N, P, ptr<const long long>(pairs), ptr<void>(ds),
                             ptr<void>(bs), ptr<void>(q), nullptr, kappa, ke, ptr<double>(E_real), ptr<void>(gds),
                             ptr<void>(gq), nullptr, st),
            "real-space pair energy");
    if (kspace && N > 0) {
      const size_t nbytes = admp_pme_recip_workspace_size(dt, (int)nf, km.data());
      TORCH_CHECK(nbytes > 0, "reciprocal workspace: ", admp_last_error_message());
      Tensor ws = torch::empty({(int64_t)nbytes}, pos.options().dtype(torch::kUInt8));
      check(admp_pme_recip(dt, (int)nf, (int)N, km.data(), ptr<void>(pos), ptr<void>(box), ptr<void>(q), kappa, ke,
                           ptr<double>(E_recip), ptr<void>(gpos), ptr<void>(gq), ptr<void>(gbox), ptr<void>(ws),
                           nbytes, st),
            "reciprocal PME");
    }
    int flags = 0;
    if (kspace) flags |= ADMP_TERM_SELF | ADMP_TERM_NON_NEUTRAL;
    if (slab) flags |= ADMP_TERM_SLAB | ((int)axis << 8);
    if (flags && N > 0)
      check(admp_atom_terms(dt, flags, (int)nf, (int)N, ptr<void>(pos), ptr<void>(box), ptr<void>(q), nullptr,
                            nullptr, nullptr, kappa, ke, nullptr, ptr<double>(terms), ptr<void>(gq), ptr<void>(gpos),
                            ptr<void>(gbox), nullptr, nullptr, nullptr, st),
            "self / non-neutral / slab terms");
    Tensor comps = torch::stack({E_real, E_recip, terms.select(1, 0), terms.select(1, 1), terms.select(1, 2)}, 1);
    Tensor E = comps.sum(1).to(q.scalar_type());
    Tensor kmt = torch::tensor(std::vector<int64_t>(km.begin(), km.end()), torch::kLong).reshape({nf, 3});
    ctx->save_for_backward({gpos, gbox, gds, gq});
    ctx->mark_non_differentiable({comps, kmt});
    return {E, comps, kmt};
  }

  static variable_list backward(AutogradContext* ctx, variable_list g) {
    auto s = ctx->get_saved_variables();
    const Tensor& gE = g[0];
    Tensor out_pos, out_box, out_ds, out_q;
    if (gE.defined() && s[3].defined()) {
      const Tensor w = gE.to(s[3].scalar_type());
      out_pos = s[0] * w.view({-1, 1, 1});
      out_box = s[1] * w.view({-1, 1, 1});
      out_ds = s[2] * w.view({-1, 1});
      out_q = s[3] * w.view({-1, 1});
    }
    return {out_pos, out_box, out_ds, out_q, Tensor(), Tensor(), Tensor(), Tensor(), Tensor(), Tensor(),
            Tensor(), Tensor(), Tensor(), Tensor(), Tensor()};
  }
};

class CoulombOBC : public torch::autograd::Function<CoulombOBC> {
 public:
  static variable_list forward(AutogradContext* ctx, Tensor ds, Tensor q, Tensor pairs, Tensor bs, double ke) {
    const int dt = dtype_code(q);
    void* st = stream_of(q);
    const int64_t nf = q.size(0), N = q.size(1), P = pairs.size(1);
    const bool need = ds.requires_grad() || q.requires_grad();
    Tensor E = f64(nf, q), gds, gq;
    if (need) {
      gds = torch::zeros_like(ds);
      gq = torch::zeros_like(q);
    }
    if (P > 0)
      check(admp_pair_energy(dt, ADMP_PAIR_OBC, (int)nf, (int)N, P, ptr<const long long>(pairs), ptr<void>(ds),
                             ptr<void>(bs), ptr<void>(q), nullptr, 0.0, ke, ptr<double>(E), ptr<void>(gds),
                             ptr<void>(gq), nullptr, st),
            "open-boundary Coulomb");
    ctx->save_for_backward({gds, gq});
    return {E.to(q.scalar_type())};
  }

  static variable_list backward(AutogradContext* ctx, variable_list g) {
    auto s = ctx->get_saved_variables();
    Tensor out_ds, out_q;
    if (g[0].defined() && s[1].defined()) {
      const Tensor w = g[0].to(s[1].scalar_type()).view({-1, 1});
      out_ds = s[0] * w;
      out_q = s[1] * w;
    }
    return {out_ds, out_q, Tensor(), Tensor(), Tensor()};
  }
};

class Damping : public torch::autograd::Function<Damping> {
 public:
  static variable_list forward(AutogradContext* ctx, Tensor ds, Tensor q, Tensor eta, Tensor pairs, Tensor bs,
                               double ke) {
    const int dt = dtype_code(q);
    void* st = stream_of(q);
    const int64_t nf = q.size(0), N = q.size(1), P = pairs.size(1);
    const bool need = ds.requires_grad() || q.requires_grad() || eta.requires_grad();
    Tensor E = f64(nf, q), gds, gq, geta;
    if (need) {
      gds = torch::zeros_like(ds);
      gq = torch::zeros_like(q);
      geta = torch::zeros_like(eta);
    }
    if (P > 0)
      check(admp_pair_energy(dt, ADMP_PAIR_DAMPING, (int)nf, (int)N, P, ptr<const long long>(pairs), ptr<void>(ds),
                             ptr<void>(bs), ptr<void>(q), ptr<void>(eta), 0.0, ke, ptr<double>(E), ptr<void>(gds),
                             ptr<void>(gq), ptr<void>(geta), st),
            "damping pair energy");
    if (N > 0)
      check(admp_atom_terms(dt, ADMP_TERM_DAMP_SELF, (int)nf, (int)N, nullptr, nullptr, ptr<void>(q), ptr<void>(eta),
                            nullptr, nullptr, 0.0, ke, ptr<double>(E), nullptr, ptr<void>(gq), nullptr, nullptr,
                            ptr<void>(geta), nullptr, nullptr, st),
            "damping self energy");
    ctx->save_for_backward({gds, gq, geta});
    return {E.to(q.scalar_type())};
  }

  static variable_list backward(AutogradContext* ctx, variable_list g) {
    auto s = ctx->get_saved_variables();
    Tensor a, b, c;
    if (g[0].defined() && s[1].defined()) {
      const Tensor w = g[0].to(s[1].scalar_type()).view({-1, 1});
      a = s[0] * w;
      b = s[1] * w;
      c = s[2] * w;
    }
    return {a, b, c, Tensor(), Tensor(), Tensor()};
  }
};

class Site : public torch::autograd::Function<Site> {
 public:
  static variable_list forward(AutogradContext* ctx, Tensor q, Tensor chi, Tensor hard) {
    const int dt = dtype_code(q);
    void* st = stream_of(q);
    const int64_t nf = q.size(0), N = q.size(1);
    const bool need = q.requires_grad() || chi.requires_grad() || hard.requires_grad();
    Tensor E = f64(nf, q), gq, gc, gh;
    if (need) {
      gq = torch::zeros_like(q);
      gc = torch::zeros_like(chi);
      gh = torch::zeros_like(hard);
    }
    if (N > 0)
      check(admp_atom_terms(dt, ADMP_TERM_SITE, (int)nf, (int)N, nullptr, nullptr, ptr<void>(q), nullptr,
                            ptr<void>(chi), ptr<void>(hard), 0.0, 0.0, ptr<double>(E), nullptr, ptr<void>(gq), nullptr,
                            nullptr, nullptr, ptr<void>(gc), ptr<void>(gh), st),
            "site energy");
    ctx->save_for_backward({gq, gc, gh});
    return {E.to(q.scalar_type())};
  }

  static variable_list backward(AutogradContext* ctx, variable_list g) {
    auto s = ctx->get_saved_variables();
    Tensor a, b, c;
    if (g[0].defined() && s[0].defined()) {
      const Tensor w = g[0].to(s[0].scalar_type()).view({-1, 1});
      a = s[0] * w;
      b = s[1] * w;
      c = s[2] * w;
    }
    return {a, b, c};
  }
};

std::vector<Tensor> coulomb_pbc(Tensor pos, Tensor box, Tensor pairs, Tensor ds, Tensor bs, Tensor q, double kappa,
                                std::vector<int64_t> kmesh, std::vector<double> spacing, double ethresh, double ke,
                                bool rspace, bool kspace, bool slab, int64_t axis) {
  TORCH_CHECK(kmesh.empty() || kmesh.size() == 3, "kmesh: 3 values or none");
  TORCH_CHECK(spacing.empty() || spacing.size() == 3, "spacing: 3 values or none");
  auto r = CoulombPBC::apply(pos.contiguous(), box.contiguous(), ds.contiguous(), q.contiguous(),
                             pairs.to(torch::kLong).contiguous(), bs.contiguous(), kappa, kmesh, spacing, ethresh, ke,
                             rspace, kspace, slab, axis);
  return {r[0], r[1], r[2]};
}

Tensor coulomb_obc(Tensor pairs, Tensor ds, Tensor bs, Tensor q, double ke) {
  return CoulombOBC::apply(ds.contiguous(), q.contiguous(), pairs.to(torch::kLong).contiguous(), bs.contiguous(),
                           ke)[0];
}

Tensor damping(Tensor ds, Tensor q, Tensor eta, Tensor pairs, Tensor bs, double ke) {
  return Damping::apply(ds.contiguous(), q.contiguous(), eta.contiguous(), pairs.to(torch::kLong).contiguous(),
                        bs.contiguous(), ke)[0];
}

Tensor site(Tensor q, Tensor chi, Tensor hard) {
  return Site::apply(q.contiguous(), chi.contiguous(), hard.contiguous())[0];
}

}  // namespace

TORCH_LIBRARY(admp_b200, m) {
  m.def("coulomb_pbc(Tensor pos, Tensor box, Tensor pairs, Tensor ds, Tensor bs, Tensor q, float kappa, "
        "int[] kmesh, float[] spacing, float ethresh, float ke, bool rspace, bool kspace, bool slab, int axis) "
        "-> Tensor[]",
        &coulomb_pbc);
  m.def("coulomb_obc(Tensor pairs, Tensor ds, Tensor bs, Tensor q, float ke) -> Tensor", &coulomb_obc);
  m.def("damping(Tensor ds, Tensor q, Tensor eta, Tensor pairs, Tensor bs, float ke) -> Tensor", &damping);
  m.def("site(Tensor q, Tensor chi, Tensor hardness) -> Tensor", &site);
}
