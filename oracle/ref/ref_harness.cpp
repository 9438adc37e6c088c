// CPU checker: the reference's own iSVD stages (MCNLA 0.7.2, header-only),
// compiled unmodified against a one-rank MPI stub and a system OpenBLAS, and
// exposed through a small C ABI so tests and the CPU-baseline leg of the bench
// can call them with plain host buffers.  This file is test infrastructure:
// nothing in the product links it.
//
// Every entry point follows the stage usage of the reference's drivers and
// tests: build Parameters (src/isvd_dense_rb.cpp:118-120), construct the stage,
// initialize(), run, read results.  Omega is passed in explicitly and the
// sketch is the same single GEMM the Gaussian-projection sketcher performs
// (include/mcnla/isvd/sketcher/gaussian_projection_sketcher.hpp:96), so the
// reference's thread-count-dependent random stream never enters a comparison.
//
// Layout conventions (all host pointers, all double):
//   A      m x n, row-major (a_colmajor = 0) or column-major (a_colmajor = 1)
//   Omega  n x (N*l), row-major
//   Q/Y    m x (N*l), row-major; sketch i owns columns [i*l, (i+1)*l)
//   Qbar   m x l, row-major
//   S      k; U m x k row-major; V n x k row-major

#include <limits>
#include <cstring>
#include <functional>
#include <memory>
#include <mcnla/isvd.hpp>

extern "C" void openblas_set_num_threads(int);
extern "C" int openblas_get_num_threads(void);

namespace {

using Val = double;
using mcnla::index_t;
using Params = mcnla::isvd::Parameters<Val>;

Params make_params(index_t m, index_t n, index_t k, index_t p, index_t N) {
  Params params(0, MPI_COMM_WORLD);
  params.setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N);
  params.sync();
  return params;
}

template <class Mat>
void load_rowmajor(Mat& dst, const Val* src, index_t m, index_t n) {
  for (index_t i = 0; i < m; ++i)
    for (index_t j = 0; j < n; ++j) dst(i, j) = src[(size_t)i * n + j];
}
template <class Mat>
void load_colmajor(Mat& dst, const Val* src, index_t m, index_t n) {
  for (index_t j = 0; j < n; ++j)
    for (index_t i = 0; i < m; ++i) dst(i, j) = src[(size_t)j * m + i];
}
template <class Mat>
void store_rowmajor(const Mat& src, Val* dst, index_t m, index_t n) {
  for (index_t i = 0; i < m; ++i)
    for (index_t j = 0; j < n; ++j) dst[(size_t)i * n + j] = src(i, j);
}

// t[0] = the stage's time(); t[1..7] = its times() parts (StageWrapper,
// include/mcnla/isvd/core/stage_wrapper.hpp:115-135).
template <class Stage>
void put_time(const Stage& s, double* t) {
  if (!t) return;
  t[0] = s.time();
  auto parts = s.times();
  for (size_t i = 0; i < parts.size() && i < 7; ++i) t[1 + i] = parts[i];
}

}  // namespace

extern "C" {

void mref_set_threads(int n) { openblas_set_num_threads(n); }
int mref_get_threads(void) { return openblas_get_num_threads(); }

// Y := A * Omega  (one GEMM on the unfolded collection).
int mref_sketch(const Val* A, int a_colmajor, int m, int n, const Val* omega, int L, Val* Y, double* t) {
  mcnla::matrix::DenseMatrixRowMajor<Val> om(n, L), y(m, L);
  load_rowmajor(om, omega, n, L);
  double t0 = mcnla::utility::getTime();
  if (a_colmajor) {
    mcnla::matrix::DenseMatrixColMajor<Val> a(m, n);
    load_colmajor(a, A, m, n);
    t0 = mcnla::utility::getTime();
    mcnla::la::mm(a, om, y);
  } else {
    mcnla::matrix::DenseMatrixRowMajor<Val> a(m, n);
    load_rowmajor(a, A, m, n);
    t0 = mcnla::utility::getTime();
    mcnla::la::mm(a, om, y);
  }
  if (t) *t = mcnla::utility::getTime() - t0;
  store_rowmajor(y, Y, m, L);
  return 0;
}

// Gramian orthogonalizer, in place on Q (m x N*l).  row_block selects
// RowBlockGramianOrthogonalizer instead of GramianOrthogonalizer.
int mref_orthogonalize(Val* Q, int m, int l, int N, int row_block, double* t) {
  auto params = make_params(m, l, l, 0, N);
  auto q = params.createCollectionQ();
  if (row_block) q = params.createCollectionQj();
  load_rowmajor(q.unfold(), Q, m, N * l);
  if (row_block) {
    mcnla::isvd::RowBlockGramianOrthogonalizer<Val> orth(params);
    orth.initialize(); orth(q); put_time(orth, t);
  } else {
    mcnla::isvd::GramianOrthogonalizer<Val> orth(params);
    orth.initialize(); orth(q); put_time(orth, t);
  }
  store_rowmajor(q.unfold(), Q, m, N * l);
  return 0;
}

// Integrators.  kind: 0 KolmogorovNagumo, 1 RowBlockKolmogorovNagumo,
// 2 RowBlockGramianKolmogorovNagumo, 3 RowBlockWenYin, 4 RowBlockGramianWenYin.
int mref_integrate(const Val* Qs, int m, int l, int N, int kind, int maxit, double tol, Val* Qbar,
                   int* iters, double* t) {
  auto params = make_params(m, l, l, 0, N);
  auto q = (kind == 0) ? params.createCollectionQ() : params.createCollectionQj();
  auto qbar = (kind == 0) ? params.createMatrixQbar() : params.createMatrixQbarj();
  load_rowmajor(q.unfold(), Qs, m, N * l);
  int it = -1;
  switch (kind) {
    case 0: { mcnla::isvd::KolmogorovNagumoIntegrator<Val> s(params, maxit, tol);
              s.initialize(); s(q, qbar); it = s.iteration(); put_time(s, t); break; }
    case 1: { mcnla::isvd::RowBlockKolmogorovNagumoIntegrator<Val> s(params, maxit, tol);
              s.initialize(); s(q, qbar); it = s.iteration(); put_time(s, t); break; }
    case 2: { mcnla::isvd::RowBlockGramianKolmogorovNagumoIntegrator<Val> s(params, maxit, tol);
              s.initialize(); s(q, qbar); it = s.iteration(); put_time(s, t); break; }
    case 3: { mcnla::isvd::RowBlockWenYinIntegrator<Val> s(params, maxit, tol);
              s.initialize(); s(q, qbar); it = s.iteration(); put_time(s, t); break; }
    case 4: { mcnla::isvd::RowBlockGramianWenYinIntegrator<Val> s(params, maxit, tol);
              s.initialize(); s(q, qbar); it = s.iteration(); put_time(s, t); break; }
    default: return -1;
  }
  store_rowmajor(qbar, Qbar, m, l);
  if (iters) *iters = it;
  return 0;
}

// Formers (all with V).  kind: 0 SvdFormer, 1 GramianFormer,
// 2 RowBlockGramianFormer, 3 ColBlockGramianFormer (A column-major).
int mref_form(const Val* A, int a_colmajor, int m, int n, const Val* Qbar, int k, int p, int kind,
              Val* S, Val* U, Val* V, double* t) {
  auto params = make_params(m, n, k, p, 1);
  const int l = k + p;
  auto qbar = params.createMatrixQbar();
  load_rowmajor(qbar, Qbar, m, l);
  auto run = [&](auto& former, auto& a) {
    former.initialize(); former(a, qbar); put_time(former, t);
    const auto& s = former.vectorS();
    for (int i = 0; i < k; ++i) S[i] = s(i);
  };
  if (kind == 3 || a_colmajor) {
    mcnla::matrix::DenseMatrixColMajor<Val> a(m, n);
    load_colmajor(a, A, m, n);
    if (kind == 3) {
      mcnla::isvd::ColBlockGramianFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixU(), U, m, k); store_rowmajor(f.matrixVj(), V, n, k);
    } else if (kind == 0) {
      mcnla::isvd::SvdFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixU(), U, m, k); store_rowmajor(f.matrixV(), V, n, k);
    } else if (kind == 1) {
      mcnla::isvd::GramianFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixU(), U, m, k); store_rowmajor(f.matrixV(), V, n, k);
    } else {
      return -1;
    }
  } else {
    mcnla::matrix::DenseMatrixRowMajor<Val> a(m, n);
    load_rowmajor(a, A, m, n);
    if (kind == 0) {
      mcnla::isvd::SvdFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixU(), U, m, k); store_rowmajor(f.matrixV(), V, n, k);
    } else if (kind == 1) {
      mcnla::isvd::GramianFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixU(), U, m, k); store_rowmajor(f.matrixV(), V, n, k);
    } else if (kind == 2) {
      mcnla::isvd::RowBlockGramianFormer<Val, true> f(params); run(f, a);
      store_rowmajor(f.matrixUj(), U, m, k); store_rowmajor(f.matrixVj(), V, n, k);
    } else {
      return -1;
    }
  }
  return 0;
}


// ---- a whole solve held between calls, the way the reference's drivers run it
// (src/isvd_dense_rb.cpp:118-221, src/isvd_dense_cb.cpp): Parameters, the four
// stages constructed and initialize()d once, A and Omega loaded into the
// reference's own matrices once (the drivers read A from a file before
// timing), then each mref_solver_run executes sketch -> orthogonalize ->
// integrate -> form and reports every stage's own time() (the drivers' and
// report/'s StageWrapper timers).  The sketch is the sketcher's projection
// GEMM with the explicit Omega (gaussian_projection_sketcher.hpp:96), timed
// around that GEMM alone.
//   integrator: as mref_integrate; former: as mref_form (3 needs a_colmajor);
//   row_block: RowBlockGramianOrthogonalizer instead of GramianOrthogonalizer.
struct MrefSolver {
  Params params;
  int colmajor = 0, kind = 0, fkind = 0, k = 0;
  mcnla::matrix::DenseMatrixRowMajor<Val> arm, om;
  mcnla::matrix::DenseMatrixColMajor<Val> acm;
  mcnla::matrix::DenseMatrixCollectionColBlockRowMajor<Val> q;
  mcnla::matrix::DenseMatrixRowMajor<Val> qbar;
  std::function<double()> orth, form;
  std::function<double(int*)> integ;
  std::function<void(Val*, Val*, Val*)> result;
  explicit MrefSolver(Params p) : params(std::move(p)) {}
};

void* mref_solver_create(const Val* A, int a_colmajor, int m, int n, int k, int p, int N, int row_block, int kind,
                         int fkind, int maxit, double tol, const Val* omega) {
  auto* s = new MrefSolver(make_params(m, n, k, p, N));
  s->colmajor = a_colmajor; s->kind = kind; s->fkind = fkind; s->k = k;
  const int L = (k + p) * N;
  if (a_colmajor) { s->acm.reconstruct(m, n); load_colmajor(s->acm, A, m, n); }
  else { s->arm.reconstruct(m, n); load_rowmajor(s->arm, A, m, n); }
  s->om.reconstruct(n, L);
  load_rowmajor(s->om, omega, n, L);
  s->q = kind == 0 ? s->params.createCollectionQ() : s->params.createCollectionQj();
  s->qbar = kind == 0 ? s->params.createMatrixQbar() : s->params.createMatrixQbarj();
  Params& prm = s->params;
  if (row_block) {
    auto o = std::make_shared<mcnla::isvd::RowBlockGramianOrthogonalizer<Val>>(prm);
    o->initialize();
    s->orth = [s, o] { (*o)(s->q); return o->time(); };
  } else {
    auto o = std::make_shared<mcnla::isvd::GramianOrthogonalizer<Val>>(prm);
    o->initialize();
    s->orth = [s, o] { (*o)(s->q); return o->time(); };
  }
  auto set_integ = [&](auto o) {
    o->initialize();
    s->integ = [s, o](int* it) { (*o)(s->q, s->qbar); *it = o->iteration(); return o->time(); };
  };
  switch (kind) {
    case 0: set_integ(std::make_shared<mcnla::isvd::KolmogorovNagumoIntegrator<Val>>(prm, maxit, tol)); break;
    case 1: set_integ(std::make_shared<mcnla::isvd::RowBlockKolmogorovNagumoIntegrator<Val>>(prm, maxit, tol)); break;
    case 2: set_integ(std::make_shared<mcnla::isvd::RowBlockGramianKolmogorovNagumoIntegrator<Val>>(prm, maxit, tol)); break;
    case 3: set_integ(std::make_shared<mcnla::isvd::RowBlockWenYinIntegrator<Val>>(prm, maxit, tol)); break;
    case 4: set_integ(std::make_shared<mcnla::isvd::RowBlockGramianWenYinIntegrator<Val>>(prm, maxit, tol)); break;
    default: delete s; return nullptr;
  }
  // U and V read from matrixU/matrixV (plain formers) or matrixUj/matrixVj (row-block former)
  auto uv = [s](const auto& u, const auto& v, Val* U, Val* V) {
    store_rowmajor(u, U, s->params.nrow(), s->k);
    store_rowmajor(v, V, s->params.ncol(), s->k);
  };
  auto set_form = [&](auto f, auto& a, auto store) {
    f->initialize();
    s->form = [s, f, &a] { (*f)(a, s->qbar); return f->time(); };
    s->result = [s, f, store](Val* S, Val* U, Val* V) {
      const auto& sv = f->vectorS();
      for (int i = 0; i < s->k; ++i) S[i] = sv(i);
      store(*f, U, V);
    };
  };
  auto plain = [uv](const auto& f, Val* U, Val* V) { uv(f.matrixU(), f.matrixV(), U, V); };
  auto rowblk = [uv](const auto& f, Val* U, Val* V) { uv(f.matrixUj(), f.matrixVj(), U, V); };
  auto colblk = [uv](const auto& f, Val* U, Val* V) { uv(f.matrixU(), f.matrixVj(), U, V); };
  if (a_colmajor) {
    if (fkind == 0) set_form(std::make_shared<mcnla::isvd::SvdFormer<Val, true>>(prm), s->acm, plain);
    else if (fkind == 1) set_form(std::make_shared<mcnla::isvd::GramianFormer<Val, true>>(prm), s->acm, plain);
    else if (fkind == 3) set_form(std::make_shared<mcnla::isvd::ColBlockGramianFormer<Val, true>>(prm), s->acm, colblk);
    else { delete s; return nullptr; }
  } else {
    if (fkind == 0) set_form(std::make_shared<mcnla::isvd::SvdFormer<Val, true>>(prm), s->arm, plain);
    else if (fkind == 1) set_form(std::make_shared<mcnla::isvd::GramianFormer<Val, true>>(prm), s->arm, plain);
    else if (fkind == 2) set_form(std::make_shared<mcnla::isvd::RowBlockGramianFormer<Val, true>>(prm), s->arm, rowblk);
    else { delete s; return nullptr; }
  }
  return s;
}

// t[0..3]: sketch, orthogonalize, integrate, form seconds (each stage's own timer).
int mref_solver_run(void* h, double* t, int* iters) {
  auto* s = static_cast<MrefSolver*>(h);
  if (!s) return -1;
  auto qu = s->q.unfold();
  double t0 = mcnla::utility::getTime();
  if (s->colmajor) mcnla::la::mm(s->acm, s->om, qu);
  else mcnla::la::mm(s->arm, s->om, qu);
  t[0] = mcnla::utility::getTime() - t0;
  t[1] = s->orth();
  t[2] = s->integ(iters);
  t[3] = s->form();
  return 0;
}

int mref_solver_result(void* h, Val* S, Val* U, Val* V) {
  auto* s = static_cast<MrefSolver*>(h);
  if (!s) return -1;
  s->result(S, U, V);
  return 0;
}

void mref_solver_destroy(void* h) { delete static_cast<MrefSolver*>(h); }

}  // extern "C"
