// drop_in.cpp -- Alien's OWN Krylov templates running on libab2.
//
// TEST PROGRAM.  Built by tests/cpp/Makefile from the reference sources where
// they lie (ALIEN_REF_SRC): expression/krylov/{Iteration,CG,BiCGStab,
// DiagPreconditioner,ChebyshevPreconditioner,NeumannPolyPreconditioner}.h,
// included unmodified.  The
// algebra they are instantiated with is Alien::B200::Algebra
// (include/alien/b200/B200Algebra.h): every vector operation, SpMV, dot
// product and preconditioner application runs on the GPU through the C ABI.
// ILU(0) is Alien::B200::ILU0Preconditioner (the reference's runs on host
// arrays), FILU0 Alien::B200::FILU0Preconditioner likewise.  The only stand-in supplied here is the ITraceMng the templates
// take a pointer to (Arccore is not available).
//
//   drop_in <dir> <cg|bicgs> <diag|ilu0|cheb|cheb_saad|neumann|filu0> <tol> <max_iter> [solve2]
//
// reads <dir>/{rp.i32,ci.i32,v.f64,b.f64} (n = size of b), solves from x = 0,
// writes <dir>/x.f64 and prints one JSON line with the iteration count, the
// status, the breakdown (if any) and the number of GPU kernel launches.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <ostream>
#include <string>
#include <vector>

#include <alien/b200/B200Algebra.h>

namespace Alien {
class ITraceMng {
 public:
  std::ostream& info() {
    static std::ostream sink(nullptr);
    return sink;
  }
};
}  // namespace Alien

#include <alien/expression/krylov/Iteration.h>
#include <alien/expression/krylov/CG.h>
#include <alien/expression/krylov/BiCGStab.h>
#include <alien/expression/krylov/DiagPreconditioner.h>
#include <alien/expression/krylov/ChebyshevPreconditioner.h>
#include <alien/expression/krylov/NeumannPolyPreconditioner.h>

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

using Algebra = Alien::B200::Algebra;

}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    std::cerr << "usage: drop_in <dir> <cg|bicgs> <diag|ilu0|cheb|cheb_saad> <tol> <max_iter> [solve2]\n";
    return 2;
  }
  const std::string dir = argv[1], solver = argv[2], pc_name = argv[3];
  const double tol = std::atof(argv[4]);
  const int max_iter = std::atoi(argv[5]);
  const bool use_solve2 = argc > 6 && std::string(argv[6]) == "solve2";
  const auto rp = read_all<int>(dir + "/rp.i32");
  const auto ci = read_all<int>(dir + "/ci.i32");
  const auto v = read_all<double>(dir + "/v.f64");
  const auto bh = read_all<double>(dir + "/b.f64");
  const int n = (int)bh.size();

  Alien::B200::Context ctx(0);
  Alien::B200::Matrix A(ctx, n, rp.data(), ci.data(), v.data());
  Alien::B200::Vector b(ctx, n), x(ctx, n);
  b.upload(bh.data());
  Algebra alg(ctx);
  alg.assign(x, 0.0);
  Alien::ITraceMng trace;
  long long launches0 = 0, launches1 = 0;
  ab2_context_launch_count(ctx.handle(), &launches0);

  Alien::Iteration<Algebra> it(alg, b, tol, max_iter, nullptr);
  std::string breakdown = "null";
  auto run = [&](auto& pc) {
    try {
      if (solver == "cg") {
        Alien::CG<Algebra> s(alg, nullptr);
        if (use_solve2) s.solve2(pc, it, A, b, x);
        else s.solve(pc, it, A, b, x);
      } else {
        Alien::BiCGStab<Algebra> s(alg, nullptr);
        if (use_solve2) s.solve2(pc, it, A, b, x);
        else s.solve(pc, it, A, b, x);
      }
    } catch (Algebra::NullValueException const& e) {
      breakdown = "\"" + e.which + "\"";
    }
  };
  if (pc_name == "diag") {
    Alien::DiagPreconditioner<Algebra> pc(alg, A);
    pc.init();
    run(pc);
  } else if (pc_name == "ilu0") {
    Alien::B200::ILU0Preconditioner<Algebra> pc(alg, A);
    pc.init();
    run(pc);
  } else if (pc_name == "cheb") {
    Alien::ChebyshevPreconditioner<Algebra> pc(alg, A, 0.0, 3, 20, nullptr);
    pc.init();
    run(pc);
  } else if (pc_name == "cheb_saad") {
    Alien::ChebyshevPreconditioner<Algebra, true> pc(alg, A, 0.0, 3, 20, &trace);
    pc.init();
    run(pc);
  } else if (pc_name == "neumann") {
    // omega from dir/omega.txt: the template's own estimate seeds from std::random_device
    double omega = 0.0;
    std::ifstream(dir + "/omega.txt") >> omega;
    Alien::NeumannPolyPreconditioner<Algebra> pc(alg, A, omega, 3, 20, nullptr);
    pc.init();
    run(pc);
  } else if (pc_name == "filu0") {
    Alien::B200::FILU0Preconditioner<Algebra> pc(alg, A);
    pc.setParameter("nb-factor-iter", 0);
    pc.setParameter("nb-solver-iter", 3);
    pc.init();
    run(pc);
  } else {
    std::cerr << "unknown preconditioner " << pc_name << "\n";
    return 2;
  }
  ab2_context_launch_count(ctx.handle(), &launches1);
  const std::vector<double> xh = x.download();
  std::ofstream(dir + "/x.f64", std::ios::binary).write(reinterpret_cast<const char*>(xh.data()),
                                                          (std::streamsize)(sizeof(double) * xh.size()));
  std::printf("{\"iterations\": %d, \"converged\": %s, \"breakdown\": %s, \"gpu_launches\": %lld}\n", it(),
              it.getStatus() ? "true" : "false", breakdown.c_str(), launches1 - launches0);
  return 0;
}
