// lambda.cu -- the Lambda equations (PROGRAM VLAMCC, lambda/vlamcc.F:597-927)
// and the CCSD one-particle density (dens/densoo.F, densvv.F, densvo.F) as
// hand-written backward passes of the CCSD residual.
//
// With the CC equations written r(T) = Z(T) - D o T = 0 (Z: everything but the
// diagonal Fock terms, D: orbital-energy denominators) and the energy E(T),
// the Lagrangian L = E + lambda . r is stationary in T when
//   lambda = (dE/dT + (dZ/dT)^T lambda) / D,
// iterated here with the same FP64 NEWT2 division, symmetrisation and DIIS
// machinery as the amplitudes (lambda/vlamcc.F uses NEWT2 and DODIIS0 the same
// way, lambda/vlamcc.F:756,812).  (dZ/dT)^T lambda is the reverse replay of a
// recorded residual pass at the converged T (adjoint.cu).
//
// The one-particle density of the fixed-orbital Lagrangian is D_pq = dL/df_pq:
// the adjoints of the Fock blocks recorded in the residual, plus dE/df_ia =
// 2 t_i^a, plus the denominator terms of the diagonal, so that for a
// one-electron perturbation f -> f + x h' the derivative dE/dx = Tr(D h').
#include <cmath>

#include "engine.cuh"

namespace acesb200 {

int CCEngine::record_residual(bool fock_active) {
  // the forward values the previous tape's backward pass cached may change
  tape_cache_clear();
  tape.clear();
  active.clear();
  active.push_back(&X);
  if (fock_active) {
    active.push_back(&offv);
    active.push_back(&offo);
    active.push_back(&fov);
    active.push_back(&fovT);
  }
  // <ab|cd> = <cd|ab> for real orbitals: the vvvv matrix is its own transpose
  symmetric.assign(1, I_vvvv.p);
  recording = true;
  int s = residual();
  recording = false;
  return s;
}

int CCEngine::lambda_rhs() {
  const long long ov = (long long)o * v, len = ov + (long long)o * o * v * v;
  zero_adjoints();
  double *z1b = adj(Z1.p), *z2b = adj(Z2.p);
  if (!z1b || !z2b) return ACES_ERR_NOMEM;
  launch_axpy(z1b, L.p, 1.0, ov, st);
  launch_axpy(z2b, L.p + ov, 1.0, len - ov, st);
  ACES_TRY(backward());
  double *xb = adj(X.p);
  ACES_TRY(alloc(lrhs, len));
  ACES_CUDA(cudaMemcpyAsync(lrhs.p, gE.p, len * 8, cudaMemcpyDeviceToDevice, st));
  launch_axpy(lrhs.p, xb, 1.0, len, st);
  ACES_CUDA(cudaGetLastError());
  return ACES_OK;
}

int CCEngine::density(std::vector<double> &D) {
  const long long ov = (long long)o * v, len = ov + (long long)o * o * v * v;
  ACES_TRY(record_residual(true));
  zero_adjoints();
  double *z1b = adj(Z1.p), *z2b = adj(Z2.p);
  if (!z1b || !z2b) return ACES_ERR_NOMEM;
  launch_axpy(z1b, L.p, 1.0, ov, st);
  launch_axpy(z2b, L.p + ov, 1.0, len - ov, st);
  ACES_TRY(backward());
  std::vector<double> aoo((size_t)o * o), avv((size_t)v * v), aov((size_t)ov), avo((size_t)ov),
      t(len), l(len);
  ACES_CUDA(cudaMemcpyAsync(aoo.data(), adj(offo.p), aoo.size() * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(avv.data(), adj(offv.p), avv.size() * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(aov.data(), adj(fov.p), aov.size() * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(avo.data(), adj(fovT.p), avo.size() * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(t.data(), X.p, len * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaMemcpyAsync(l.data(), L.p, len * 8, cudaMemcpyDeviceToHost, st));
  ACES_CUDA(cudaStreamSynchronize(st));
  D.assign((size_t)nmo * nmo, 0.0);
  auto at = [&](int p, int q) -> double & { return D[(size_t)p * nmo + q]; };
  for (int i = 0; i < o; ++i)
    for (int j = 0; j < o; ++j)
      if (i != j) at(i, j) = aoo[(size_t)i * o + j];
  for (int a = 0; a < v; ++a)
    for (int b = 0; b < v; ++b)
      if (a != b) at(o + a, o + b) = avv[(size_t)a * v + b];
  for (int i = 0; i < o; ++i)
    for (int a = 0; a < v; ++a)
      at(i, o + a) = aov[(size_t)i * v + a] + avo[(size_t)a * o + i] + 2.0 * t[(size_t)i * v + a];
  // diagonal: -lambda . d(D o T)/d e_p
  const double *t1 = t.data(), *l1 = l.data(), *t2 = t.data() + ov, *l2 = l.data() + ov;
  std::vector<double> occ(o, 0.0), vir(v, 0.0);
  for (int i = 0; i < o; ++i)
    for (int a = 0; a < v; ++a) {
      double x = l1[(size_t)i * v + a] * t1[(size_t)i * v + a];
      occ[i] -= x;
      vir[a] += x;
    }
  for (int i = 0; i < o; ++i)
    for (int j = 0; j < o; ++j)
      for (int a = 0; a < v; ++a)
        for (int b = 0; b < v; ++b) {
          size_t k = (((size_t)i * o + j) * v + a) * v + b;
          double x = l2[k] * t2[k];
          occ[i] -= x;
          occ[j] -= x;
          vir[a] += x;
          vir[b] += x;
        }
  for (int i = 0; i < o; ++i) at(i, i) = occ[i];
  for (int a = 0; a < v; ++a) at(o + a, o + a) = vir[a];
  return ACES_OK;
}

}  // namespace acesb200

using namespace acesb200;

extern "C" int xlambda_run(aces_cc_config *cfg) {
  if (!cfg) return ACES_ERR_ARG;
  State &stt = state();
  std::lock_guard<std::recursive_mutex> lk(stt.mu);
  CCEngine *Ep = engine_instance(false);
  if (!Ep || !Ep->have_amplitudes) {
    set_error("xlambda_run: no converged CC amplitudes (run xvcc_run first)");
    return ACES_ERR_ARG;
  }
  if (cfg->cc_exporder < 1 || cfg->cc_exporder > 25 || cfg->cc_maxcyc < 1) {
    set_error("xlambda_run: cc_exporder must be 1..25 and cc_maxcyc >= 1");
    return ACES_ERR_ARG;
  }
  CCEngine &E = *Ep;
  E.prec = cfg->precision;
  const long long O = E.o, V = E.v, ov = O * V, len = ov + O * O * V * V;
  ACES_TRY(E.alloc(E.L, len));
  ACES_TRY(E.alloc(E.Ln, len));
  ACES_TRY(E.alloc(E.gE, len));
  // dE/dT: dE/dt2 = 2<ij|ab> - <ij|ba>; dE/dt1 = 2 f_ia + 2 sum_jb L_ijab t_jb
  ACES_TRY(E.record_residual(false));
  ACES_CUDA(cudaMemcpyAsync(E.gE.p + ov, E.L_oovv.p, (len - ov) * 8, cudaMemcpyDeviceToDevice,
                            E.st));
  ACES_CUDA(cudaMemcpyAsync(E.gE.p, E.fov.p, ov * 8, cudaMemcpyDeviceToDevice, E.st));
  launch_scale(E.gE.p, 2.0, ov, E.st);
  ACES_TRY(E.G(E.o * E.v, 1, E.o * E.v, 2.0, E.LmeP.p, ov, E.t1(), ov, 1.0,
               cview_rowmajor(E.gE.p, 1)));
  // initial multipliers: lambda = (dE/dT) / D
  launch_newt(E.L.p + ov, E.gE.p + ov, E.L.p, E.gE.p, E.eo.p, E.ev.p, E.o, E.v, E.st);
  ACES_CUDA(cudaGetLastError());
  for (auto &b : E.hx) if (b.p) dev_free(b.p);
  for (auto &b : E.he) if (b.p) dev_free(b.p);
  E.hx.clear();
  E.he.clear();
  E.Bh.assign(625, 0.0);
  const double tol = std::pow(10.0, -cfg->cc_conv);
  cudaEvent_t ev0, ev1;
  ACES_CUDA(cudaEventCreate(&ev0));
  ACES_CUDA(cudaEventCreate(&ev1));
  double e3[3], res = 0, dres = 0;
  bool converged = false;
  int icycle;
  float ms_total = 0.f;
  int ntimed = 0;
  for (icycle = 1; icycle <= cfg->cc_maxcyc; ++icycle) {
    bool extrap = false;
    ACES_CUDA(cudaEventRecord(ev0, E.st));
    ACES_TRY(E.iteration(icycle, cfg->cc_exporder, e3, &res, &dres, &extrap, true));
    int ndimr = icycle < cfg->cc_exporder ? icycle : cfg->cc_exporder;
    bool conv = std::fabs(res) < tol;
    if (!conv) ACES_TRY(accept_update(E, extrap, ndimr, true));
    ACES_CUDA(cudaEventRecord(ev1, E.st));
    ACES_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (icycle > cfg->timing_warmup) {
      ms_total += ms;
      ntimed++;
    }
    if (cfg->verbose)
      printf("  lambda cycle %3d  max res = % .8e  max DIIS res = % .8e  %.3f ms\n", icycle, res,
             dres, ms);
    if (conv) {
      converged = true;
      break;
    }
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (icycle > cfg->cc_maxcyc) icycle = cfg->cc_maxcyc;
  cfg->ncycle = icycle;
  cfg->converged = converged ? 1 : 0;
  cfg->last_residual = res;
  cfg->seconds_per_iter = ntimed ? ms_total * 1e-3 / ntimed : 0.0;
  // L1 -> list 190, L2(AB) -> list 146, L2(AA) -> list 144 (vcc/vcc.F:622-626 list map)
  // in the reference's convention: the engine iterates the Lagrange multipliers
  // l of its spin-adapted residual, l1 = 2 L1 and l2 = 2 L2 - L2~ (L2~: the
  // virtual indices swapped), so the lists get L1 = l1 / 2, L2 = (2 l2 + l2~) / 3
  {
    DBuf r;
    ACES_TRY(E.alloc(r, len));
    const long long st2[4] = {O * V * V, V * V, V, 1};
    int ws = E.perm(r.p, 1, 1, E.o, E.v, 0.0, {PermTerm{E.L.p, 0.5, {0, 0, V, 1}}});
    if (ws == ACES_OK)
      ws = E.perm(r.p + ov, E.o, E.o, E.v, E.v, 0.0,
                  {PermTerm{E.L.p + ov, 2.0 / 3.0, {st2[0], st2[1], st2[2], st2[3]}},
                   PermTerm{E.L.p + ov, 1.0 / 3.0, {st2[0], st2[1], st2[3], st2[2]}}});
    if (ws == ACES_OK) ws = E.write_amplitudes(r.p, r.p + ov, 190, 146, 144);
    ACES_CUDA(cudaStreamSynchronize(E.st));
    dev_free(r.p);
    ACES_TRY(ws);
  }
  if (!converged) {
    set_error("Lambda equations did not converge in %d cycles", cfg->cc_maxcyc);
    return ACES_ERR_NOCONV;
  }
  E.have_lambda = true;
  return ACES_OK;
}

extern "C" int xdens_1pdm(aces_cc_config *cfg) {
  (void)cfg;
  State &stt = state();
  std::lock_guard<std::recursive_mutex> lk(stt.mu);
  CCEngine *Ep = engine_instance(false);
  if (!Ep || !Ep->have_lambda) {
    set_error("xdens_1pdm: no converged Lambda (run xvcc_run and xlambda_run first)");
    return ACES_ERR_ARG;
  }
  std::vector<double> D;
  ACES_TRY(Ep->density(D));
  for (double x : D)
    if (!std::isfinite(x)) {
      set_error("xdens_1pdm: non-finite density");
      return ACES_ERR_NAN;
    }
  return aces_putrec("DENSMAT", (long long)D.size() * 8, D.data());
}
