// facade.cpp -- TEST PROGRAM: libab2 behind Alien's own back-end interfaces.
//
// Built by tests/cpp/Makefile against the reference's headers where they lie
// (ALIEN_REF_SRC): core/backend/{BackEnd,IInternalLinearAlgebraT,
// IInternalLinearSolverT}.h and expression/solver/{ILinearSolver,SolverStat}.h,
// with SolverStat.cc compiled from the reference too.  The only stand-ins are
// the Arccore declarations in arccore_stub/ (Arccore is not available).  Every
// call below goes through AlgebraTraits<BackEnd::tag::b200> and the virtual
// interfaces IInternalLinearAlgebra / IInternalLinearSolver, as Alien's
// LinearAlgebra<Tag> and LinearSolver<Tag> facades make them.
//
//   facade traits
//       prints the traits' name and hasParallelSupport() (no GPU needed)
//   facade algebra <dir>
//       reads <dir>/{rp.i32,ci.i32,v.f64,b.f64}, converts them as the
//       simplecsr -> b200 converters do, and writes <dir>/out_*.f64: mult,
//       axpy, aypx, copy, scal, diagonal, reciprocal, pointwiseMult, and
//       out_scalars.f64 = {dot(b,b), norm0, norm1, norm2}
//   facade solve <dir> <cg|bicgs> <precond> <tol> <max_iter> [mixed]
//       solves A x = b from x = 0 through solver_factory(options), writes
//       <dir>/x.f64 and prints one JSON line with getStatus() and
//       getSolverStat()
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <alien/b200/backend.h>

namespace {

template <class T>
std::vector<T> read_all(const std::string& path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) {
    std::cerr << "cannot read " << path << "\n";
    std::exit(2);
  }
  const std::streamsize bytes = f.tellg();
  f.seekg(0);
  std::vector<T> v((std::size_t)bytes / sizeof(T));
  f.read(reinterpret_cast<char*>(v.data()), bytes);
  return v;
}

void write_all(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

using Traits = Alien::AlgebraTraits<Alien::BackEnd::tag::b200>;
using M = Traits::matrix_type;
using V = Traits::vector_type;

template <class T>
Arccore::ConstArrayView<T> view(const std::vector<T>& v) {
  return Arccore::ConstArrayView<T>((Arccore::Integer)v.size(), v.data());
}

struct Input {
  std::vector<int> rp, ci;
  std::vector<double> v, b;
};

Input read_input(const std::string& dir) {
  return Input{read_all<int>(dir + "/rp.i32"), read_all<int>(dir + "/ci.i32"), read_all<double>(dir + "/v.f64"),
               read_all<double>(dir + "/b.f64")};
}

std::vector<double> host(const V& x) {
  std::vector<double> out((std::size_t)x.size());
  Alien::B200::toSimpleCSR(x, Arccore::ArrayView<double>((Arccore::Integer)out.size(), out.data()));
  return out;
}

// An ITraceMng that writes info() to stderr (SolverStat::print's target).
class StderrTrace : public Arccore::ITraceMng {
 public:
  std::ostream& info() override { return std::cerr; }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: facade traits | algebra <dir> | solve <dir> <solver> <precond> <tol> <max_iter> [mixed]\n";
    return 2;
  }
  const std::string mode = argv[1];
  try {
    if (mode == "traits") {
      std::unique_ptr<Traits::solver_type> s(Traits::solver_factory());
      std::cout << "{\"name\": \"" << Traits::name() << "\", \"parallel\": " << (s->hasParallelSupport() ? 1 : 0)
                << "}" << std::endl;
      return 0;
    }
    if (argc < 3) return 2;
    const std::string dir = argv[2];
    const Input in = read_input(dir);
    const int n = (int)in.b.size();
    if (mode == "algebra") {
      std::unique_ptr<Traits::algebra_type> alg(Traits::algebra_factory());
      const auto& ctx = static_cast<Alien::B200::InternalLinearAlgebra*>(alg.get())->context();
      const M A = Alien::B200::fromSimpleCSR(ctx, view(in.rp), view(in.ci), view(in.v));
      const V b = Alien::B200::fromSimpleCSR(ctx, view(in.b));
      V y(ctx, n), z(ctx, n), d(ctx, n), w(ctx, n), c(ctx, n);
      alg->mult(A, b, y);
      write_all(dir + "/out_mult.f64", host(y));
      alg->copy(y, z);
      write_all(dir + "/out_copy.f64", host(z));
      alg->axpy(-0.75, b, z);  // z = y - 0.75 b
      write_all(dir + "/out_axpy.f64", host(z));
      alg->copy(y, c);
      alg->aypx(0.5, c, b);  // c = 0.5 y + b
      write_all(dir + "/out_aypx.f64", host(c));
      alg->scal(3.0, c);
      write_all(dir + "/out_scal.f64", host(c));
      alg->diagonal(A, d);
      write_all(dir + "/out_diagonal.f64", host(d));
      alg->reciprocal(d);
      write_all(dir + "/out_reciprocal.f64", host(d));
      alg->pointwiseMult(b, d, w);
      write_all(dir + "/out_pmult.f64", host(w));
      write_all(dir + "/out_scalars.f64", {alg->dot(b, b), alg->norm0(b), alg->norm1(b), alg->norm2(b)});
      bool dump_throws = false;
      try {
        alg->dump(A, "unused");
      } catch (const Arccore::NotImplementedException&) {
        dump_throws = true;
      }
      std::cout << "{\"dump_not_implemented\": " << (dump_throws ? 1 : 0) << "}" << std::endl;
      return 0;
    }
    if (mode == "solve" && argc >= 7) {
      Traits::options_type opts;
      opts.solver = argv[3];
      opts.precond = argv[4];
      opts.tol = std::atof(argv[5]);
      opts.max_iter = std::atoi(argv[6]);
      opts.mixed = argc > 7 && std::string(argv[7]) == "mixed";
      std::unique_ptr<Traits::solver_type> s(Traits::solver_factory(opts));
      s->init();
      Alien::B200::Context ctx(opts.device);
      const int formats = AB2_FMT_CSR | AB2_FMT_ELL | AB2_FMT_STENCIL | (opts.mixed ? AB2_FMT_F32 : 0);
      const M A = Alien::B200::fromSimpleCSR(ctx, view(in.rp), view(in.ci), view(in.v), formats);
      const V b = Alien::B200::fromSimpleCSR(ctx, view(in.b));
      V x(ctx, n);
      std::vector<double> zero((std::size_t)n, 0.0);
      x.upload(zero.data());
      const bool ok = s->solve(A, b, x);
      write_all(dir + "/x.f64", host(x));
      const Alien::SolverStatus& st = s->getStatus();
      const Alien::SolverStat& stat = s->getSolverStat();
      StderrTrace trace;
      stat.print(&trace, st, "b200");
      s->end();
      std::ostringstream o;
      o.precision(17);
      o << "{\"ok\": " << (ok ? 1 : 0) << ", \"succeeded\": " << (st.succeeded ? 1 : 0)
        << ", \"iterations\": " << st.iteration_count << ", \"residual\": " << st.residual
        << ", \"error\": " << st.error << ", \"solve_count\": " << stat.solveCount()
        << ", \"stat_iterations\": " << stat.iterationCount()
        << ", \"last_iterations\": " << stat.lastIterationCount() << ", \"solve_time\": " << stat.lastSolveTime()
        << ", \"parallel\": " << (s->hasParallelSupport() ? 1 : 0) << "}";
      std::cout << o.str() << std::endl;
      return 0;
    }
  } catch (const std::exception& e) {
    std::cerr << "facade: " << e.what() << "\n";
    return 1;
  }
  std::cerr << "facade: bad arguments\n";
  return 2;
}
