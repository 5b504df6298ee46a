// ml_prec_b200: the command-line driver of project/main.cc for the PCG path.
//
//   ml_prec_b200 -p multi_split -C msplit.cfg [-x 60 -y 220 -z 85] [-c 1]
//                [--eps 1e-8] [--dirichlet] [--fp32] [-a ntests]
//
// It builds the SPE matrix (or loads -m/-v files), constructs the
// preconditioner ntests times, solves ntests times, and prints the
// construction and solution times and the iteration count. When the working
// directory holds default.properties, the log4j.appender.R.File key names a
// file (inside --dir) that receives the same log lines.
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <fstream>
#include <memory>

#include "ml_prec.h"

namespace {

struct Log {
    std::ofstream file;
    template <class T>
    Log& operator<<(const T& v) {
        std::cout << v;
        if (file.is_open()) file << v;
        return *this;
    }
    Log& operator<<(std::ostream& (*f)(std::ostream&)) {
        std::cout << f;
        if (file.is_open()) file << f;
        return *this;
    }
};

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char* argv[]) {
    try {
        Config cfg;
        if (set_params(argc, argv, cfg)) {
            std::cout << "Error while setting parameters, exiting..." << std::endl;
            return 1;
        }
        Log log;
        {
            std::ifstream probe("default.properties");
            if (probe.good()) {
                ConfigFile props("default.properties");
                std::string f = props.read<std::string>("log4j.appender.R.File", "");
                if (!f.empty()) {
                    mkdir(cfg.dir.c_str(), 0755);
                    log.file.open((cfg.dir + "/" + f).c_str());
                }
            }
        }
        log << "Config parameters:\n" << cfg;

        SkylineMatrix A;
        Vector b;
        if (cfg.matrix.empty()) {
            SPEMesh mesh(cfg.nx, cfg.ny, cfg.nz, cfg.perm_file);
            if (cfg.dirichlet)
                mesh.construct_matrix_dirichlet(A, b, cfg.c);
            else
                construct_matrix(cfg, mesh, A);
        } else {
            A.load(cfg.matrix, cfg.matrix.find(".crs") != std::string::npos  ? ASCII
                               : cfg.matrix.find(".mm") != std::string::npos ? MATRIX_MARKET
                                                                              : BINARY,
                   true);
        }
        if (b.size() != A.size()) b.assign(A.size(), 0.0);
        construct_vector(cfg, b);

        if (cfg.dump_data) {
            dump("matrix.dat", A, BINARY);
            dump("vector.dat", b, BINARY);
            return 0;
        }

        std::unique_ptr<PrecBase> B;
        std::vector<double> ctimes, stimes;
        for (uint i = 0; i < cfg.ntests; i++) {
            B.reset();
            double t0 = now();
            B.reset(make_prec(A, cfg));
            ctimes.push_back(now() - t0);
            log << "Construction time : " << ctimes.back() << std::endl;
        }
        log << *dynamic_cast<DevicePrec*>(B.get());

        Vector x(A.size());
        SolverStats stats;
        for (uint i = 0; i < cfg.ntests; i++) {
            if (cfg.solver == CHEB_SOLVER) {
                // main.cc:141-149: the uh_cheb preconditioner's level-0 bounds
                const Prec& Bc = dynamic_cast<const Prec&>(*B);
                double t0 = now();
                ChebSolver(A, Bc.lmin(), Bc.lmax(), b, Bc, x, cfg.eps);
                stats.t_sol = now() - t0;
            } else {
                PCGSolver(A, b, *B, x, stats, cfg.eps);
            }
            stimes.push_back(stats.t_sol);
            log << "Solution time : " << stimes.back() << std::endl;
        }
        double tc = avg_time(ctimes), ts = avg_time(stimes);
        log << "Number of iterations : " << stats.niter << std::endl;
        log << "Final relative residual : " << stats.final_rel << std::endl;
        log << "Avg construction time: " << tc << std::endl;
        log << "Avg solution time    : " << ts << std::endl;
        log << "Avg total time       : " << tc + ts << std::endl;
        return 0;
    } catch (const Exception& e) {
        std::cerr << "Exception: " << e.what() << std::endl;
        return 2;
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << std::endl;
        return 2;
    }
}
