// dist_drop_in.cpp -- Alien's OWN Krylov templates on the row-block
// distributed algebra, R ranks in one process.
//
// TEST PROGRAM.  Built by tests/cpp/Makefile from the reference sources where
// they lie (ALIEN_REF_SRC): expression/krylov/{Iteration,CG,BiCGStab,
// DiagPreconditioner}.h, included unmodified.  Every rank runs the templates
// on its own host thread with Alien::B200::DistAlgebra
// (include/alien/b200/B200DistAlgebra.h) over a local group of ranks on one
// GPU: the SpMV exchanges ghost values, the dots are summed over the ranks,
// ILU(0) is the block-Jacobi Alien::B200::DistILU0Preconditioner -- what the
// reference's parallel SimpleCSR algebra does on R MPI ranks.
//
//   dist_drop_in <dir> <cg|bicgs> <diag|ilu0> <tol> <max_iter>
//
// reads <dir>/{rp.i32,ci.i32,v.f64,b.f64} (the global system) and
// <dir>/off.i32 (R+1 row offsets), solves from x = 0, writes <dir>/x.f64 and
// prints one JSON line: iterations and status (identical on every rank, which
// is checked), breakdown, GPU kernel launches over all ranks.
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <iostream>
#include <ostream>
#include <string>
#include <thread>
#include <vector>

#include <alien/b200/B200DistAlgebra.h>

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

using Algebra = Alien::B200::DistAlgebra;

struct RankOut {
  int iterations = -1;
  bool converged = false;
  std::string breakdown = "null";
  std::string error;
  std::vector<double> x;
  long long launches = 0;
};

}  // namespace

int main(int argc, char** argv) {
  if (argc < 6) {
    std::cerr << "usage: dist_drop_in <dir> <cg|bicgs> <diag|ilu0> <tol> <max_iter>\n";
    return 2;
  }
  const std::string dir = argv[1], solver = argv[2], pc_name = argv[3];
  const double tol = std::atof(argv[4]);
  const int max_iter = std::atoi(argv[5]);
  const auto rp = read_all<int>(dir + "/rp.i32");
  const auto ci = read_all<int>(dir + "/ci.i32");
  const auto v = read_all<double>(dir + "/v.f64");
  const auto bh = read_all<double>(dir + "/b.f64");
  const auto off = read_all<int>(dir + "/off.i32");
  const int nranks = (int)off.size() - 1;

  std::vector<Alien::B200::Context> ctxs;
  for (int r = 0; r < nranks; ++r) ctxs.emplace_back(0);
  std::vector<Alien::B200::Comm> comms = Alien::B200::Comm::localGroup(ctxs, 60.0);
  std::vector<RankOut> out((std::size_t)nranks);

  auto rank_main = [&](int r) {
    RankOut& o = out[(std::size_t)r];
    try {
      const Alien::B200::Context& ctx = ctxs[(std::size_t)r];
      long long l0 = 0, l1 = 0;
      ab2_context_launch_count(ctx.handle(), &l0);
      const int a = off[(std::size_t)r], e = off[(std::size_t)r + 1];
      std::vector<int> lrp((std::size_t)(e - a) + 1);
      for (int i = a; i <= e; ++i) lrp[(std::size_t)(i - a)] = rp[(std::size_t)i] - rp[(std::size_t)a];
      Alien::B200::DistMatrix A(ctx, comms[(std::size_t)r], off.data(), lrp.data(), ci.data() + rp[(std::size_t)a],
                                v.data() + rp[(std::size_t)a]);
      Algebra alg(ctx, comms[(std::size_t)r]);
      Alien::B200::Vector b, x;
      alg.allocate(Algebra::resource(A), b, x);
      b.upload(bh.data() + a);
      alg.assign(x, 0.0);
      Alien::ITraceMng trace;
      Alien::Iteration<Algebra> it(alg, b, tol, max_iter, nullptr);
      auto run = [&](auto& pc) {
        try {
          if (solver == "cg") {
            Alien::CG<Algebra> s(alg, nullptr);
            s.solve(pc, it, A, b, x);
          } else {
            Alien::BiCGStab<Algebra> s(alg, nullptr);
            s.solve(pc, it, A, b, x);
          }
        } catch (Algebra::NullValueException const& ex) {
          o.breakdown = "\"" + ex.which + "\"";
        }
      };
      if (pc_name == "diag") {
        Alien::DiagPreconditioner<Algebra> pc(alg, A);
        pc.init();
        run(pc);
      } else if (pc_name == "ilu0") {
        Alien::B200::DistILU0Preconditioner<Algebra> pc(alg, A);
        pc.init();
        run(pc);
      } else {
        throw std::runtime_error("unknown preconditioner " + pc_name);
      }
      ab2_context_launch_count(ctx.handle(), &l1);
      o.iterations = it();
      o.converged = it.getStatus();
      o.x = x.download();
      o.launches = l1 - l0;
    } catch (std::exception const& ex) {
      o.error = ex.what();
    }
  };
  std::vector<std::thread> threads;
  for (int r = 0; r < nranks; ++r) threads.emplace_back(rank_main, r);
  for (auto& t : threads) t.join();

  std::vector<double> xg;
  long long launches = 0;
  for (int r = 0; r < nranks; ++r) {
    const RankOut& o = out[(std::size_t)r];
    if (!o.error.empty()) {
      std::cerr << "rank " << r << ": " << o.error << "\n";
      return 1;
    }
    if (o.iterations != out[0].iterations || o.converged != out[0].converged || o.breakdown != out[0].breakdown) {
      std::cerr << "rank " << r << " disagrees with rank 0\n";
      return 1;
    }
    xg.insert(xg.end(), o.x.begin(), o.x.end());
    launches += o.launches;
  }
  std::ofstream(dir + "/x.f64", std::ios::binary).write(reinterpret_cast<const char*>(xg.data()),
                                                          (std::streamsize)(sizeof(double) * xg.size()));
  std::printf("{\"iterations\": %d, \"converged\": %s, \"breakdown\": %s, \"gpu_launches\": %lld, \"ranks\": %d}\n",
              out[0].iterations, out[0].converged ? "true" : "false", out[0].breakdown.c_str(), launches, nranks);
  return 0;
}
