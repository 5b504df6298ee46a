// Test program for the C++ host interface (ml_prec_b200/host/ml_prec.h), the
// way a program written against the reference uses it.
//
//   host_api_test cpu <tmpdir>
//       host logic only, no GPU: ConfigFile parsing, command-line parsing,
//       matrix and vector file formats, the skyline transform, configuration
//       errors raised before any device call. Prints "ok" on success.
//   host_api_test ref-files <dir>
//       files written by the reference's own writers (csrmatrix.cc:302-355,
//       vector.cc:18-49; oracle/ref/ref_driver --dump-formats) load into the
//       same matrix and vector as the raw arrays beside them (A0.csr, b.f64);
//       the reference's BINARY vector file is refused with a message. No GPU.
//   host_api_test solve <nx> <ny> <nz> <perm.bin> <cfg> <eps> <fp32> <x.bin>
//       SPEMesh + Dirichlet matrix, MultiSplitPrec(A, cfg) from the config
//       file, PCGSolver; writes x (BINARY vector format) and prints
//       "niter <n> rel <r>".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <memory>

#include "ml_prec.h"

#define CHECK(cond)                                                             \
    do {                                                                        \
        if (!(cond)) {                                                          \
            std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
            std::exit(1);                                                       \
        }                                                                       \
    } while (0)

template <class F>
static bool throws(F f, const char* needle) {
    try {
        f();
    } catch (const Exception& e) {
        if (std::string(e.what()).find(needle) != std::string::npos) return true;
        std::fprintf(stderr, "unexpected message: %s\n", e.what());
        return false;
    }
    return false;
}

static int cpu(const std::string& dir) {
    // ConfigFile: comments, continuation lines, later keys override, sentry
    {
        std::ofstream f(dir + "/t.cfg");
        f << "# comment line\n"
             "q = 0.8 0.7   # per level\n"
             "level_niter = 5\n"
             "   4\n"
             "\n"
             "elim_order  = simple_1\n"
             "degree_max = 3\n"
             "degree_max = 2\n"
             "flag = no\n"
             "EndConfigFile\n"
             "max_levels = 99\n";
    }
    ConfigFile cf(dir + "/t.cfg");
    CHECK(cf.read<std::string>("q") == "0.8 0.7");
    CHECK(cf.read<std::string>("level_niter") == "5\n   4");
    CHECK(cf.read<std::string>("elim_order") == "simple_1");
    CHECK(cf.read<uint>("degree_max") == 2);
    CHECK(cf.read<uint>("max_levels", 15) == 15);  // after the sentry
    CHECK(cf.read<bool>("flag") == false);
    CHECK(!cf.keyExists("coarse_n"));
    bool missing = false;
    try {
        cf.read<int>("nothing");
    } catch (ConfigFile::key_not_found& e) {
        missing = e.key == "nothing";
    }
    CHECK(missing);
    bool absent = false;
    try {
        ConfigFile nf(dir + "/does_not_exist.cfg");
    } catch (ConfigFile::file_not_found& e) {
        absent = true;
    }
    CHECK(absent);

    // command line (main_helper.cc option letters)
    {
        const char* argv[] = {"x", "-p", "multi_split", "-C", "m.cfg", "-x", "12", "-y", "22", "-z", "6", "-c",
                              "0.5", "-s", "0.8 0.7", "-b", "5 4", "-a", "3", "--eps", "1e-8", "--fp32",
                              "--dirichlet", "-t", "no", nullptr};
        Config cfg;
        CHECK(set_params(25, const_cast<char**>(argv), cfg) == 0);
        CHECK(cfg.prec == MULTI_SPLIT_PREC && cfg.prec_conf_file == "m.cfg");
        CHECK(cfg.nx == 12 && cfg.ny == 22 && cfg.nz == 6 && cfg.c == 0.5 && cfg.ntests == 3);
        CHECK(cfg.sigmas.size() == 2 && cfg.sigmas[1] == 0.7 && cfg.niters.size() == 2 && cfg.niters[1] == 4);
        CHECK(cfg.eps == 1e-8 && cfg.fp32 && cfg.dirichlet && !cfg.use_tails);
    }
    {
        const char* argv[] = {"x", "-p", "uh_cheb", "-s", "0.5", nullptr};
        Config cfg;
        CHECK(throws([&] { set_params(5, const_cast<char**>(argv), cfg); }, "All sigmas must be > 1"));
    }
    {
        const char* argv[] = {"x", "-p", "amg", nullptr};
        Config cfg;
        CHECK(throws([&] { set_params(3, const_cast<char**>(argv), cfg); }, "Unknown prec type"));
    }

    // matrix formats and the skyline transform (diagonal moved first)
    {
        std::ofstream f(dir + "/m.crs");
        f << "# rows cols nonzeros\n3 3 7\n# row_ptr\n0\n2\n5\n7\n# col_ind\n1\n0\n0\n2\n1\n2\n1\n# value\n"
             "-1\n2\n-1\n-1\n3\n4\n-1\n";
    }
    SkylineMatrix S;
    S.load(dir + "/m.crs", ASCII, true);
    CHECK(S.size() == 3 && S.nnz() == 7);
    const uint ja_sky[] = {0, 1, 1, 0, 2, 2, 1};
    const double a_sky[] = {2, -1, 3, -1, -1, 4, -1};
    for (uint k = 0; k < 7; k++) CHECK(S.get_ja()[k] == ja_sky[k] && S.get_a()[k] == a_sky[k]);
    CHECK(S.is_symmetric());
    CHECK(S.row_sum(1) == 1.0);
    dump(dir + "/m.dat", S, BINARY);
    SkylineMatrix S2;
    S2.load(dir + "/m.dat", BINARY, false);
    CHECK(S2.get_ia() == S.get_ia() && S2.get_ja() == S.get_ja() && S2.get_a() == S.get_a());
    dump(dir + "/m.mm", S, MATRIX_MARKET);
    SkylineMatrix S3;
    S3.load(dir + "/m.mm", MATRIX_MARKET, true);
    CHECK(S3.get_ja() == S.get_ja() && S3.get_a() == S.get_a());
    {
        std::ofstream f(dir + "/bad.crs");
        f << "# rows cols nonzeros\n2 2 2\n# row_ptr\n0\n1\n2\n# col_ind\n1\n0\n# value\n1\n1\n";
    }
    SkylineMatrix Sb;
    CHECK(throws([&] { Sb.load(dir + "/bad.crs", ASCII, true); }, "No diagonal element in row 0"));

    // vector formats (BINARY keeps all n doubles)
    Vector v(5);
    for (uint i = 0; i < 5; i++) v[i] = 0.1 * i - 3;
    dump(dir + "/v.dat", v, BINARY);
    dump(dir + "/v.crs", v, ASCII);
    Vector w, u;
    load(w, dir + "/v.dat", BINARY);
    load(u, dir + "/v.crs", ASCII);
    CHECK(w == v);
    for (uint i = 0; i < 5; i++) CHECK(std::fabs(u[i] - v[i]) < 1e-15);

    // configuration errors raised before the device is touched
    Config cfg;
    cfg.prec = MULTI_SPLIT_PREC;
    cfg.prec_conf_file = dir + "/absent.cfg";
    CHECK(throws([&] { MultiSplitPrec P(S, cfg); }, "is absent"));
    {
        std::ofstream f(dir + "/bad_order.cfg");
        f << "elim_order = optimal\n";
    }
    cfg.prec_conf_file = dir + "/bad_order.cfg";
    CHECK(throws([&] { MultiSplitPrec P(S, cfg); }, "Unknown elim_order type: optimal"));
    {
        std::ofstream f(dir + "/dyn.cfg");
        f << "inner_iter = adaptive\n";
    }
    cfg.prec_conf_file = dir + "/dyn.cfg";
    CHECK(throws([&] { MultiSplitPrec P(S, cfg); }, "Unknown inner_iter type: adaptive"));
    cfg.prec_conf_file.clear();
    cfg.sigmas.assign(1, 1.5);
    CHECK(throws([&] { MultiSplitPrec P(S, cfg); }, "All sigmas must be < 1"));
    Config cc;
    cc.sigmas.assign(1, 0.9);
    CHECK(throws([&] { Prec P(S, cc); }, "All sigmas must be > 1"));
    std::vector<double> t = {3, 1, 2, 5, 4, 9};
    CHECK(avg_time(t) == (2 + 3 + 4) / 3.0);
    std::printf("ok\n");
    return 0;
}

static std::vector<char> read_all(const std::string& fn) {
    std::ifstream is(fn.c_str(), std::ios::binary);
    return std::vector<char>((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
}

static int ref_files(const std::string& dir) {
    // raw arrays: A0.csr = uint nrow, ncol, ia[nrow+1], ja[nnz], a[nnz]; b.f64 = doubles
    std::vector<char> raw = read_all(dir + "/A0.csr");
    CHECK(raw.size() >= 8);
    uint nrow, ncol;
    std::memcpy(&nrow, raw.data(), 4);
    std::memcpy(&ncol, raw.data() + 4, 4);
    std::vector<uint> ia(nrow + 1);
    std::memcpy(ia.data(), raw.data() + 8, 4 * (size_t)(nrow + 1));
    uint nnz = ia[nrow];
    std::vector<uint> ja(nnz);
    std::vector<double> a(nnz);
    std::memcpy(ja.data(), raw.data() + 8 + 4 * (size_t)(nrow + 1), 4 * (size_t)nnz);
    std::memcpy(a.data(), raw.data() + 8 + 4 * (size_t)(nrow + 1) + 4 * (size_t)nnz, 8 * (size_t)nnz);
    std::vector<char> rb = read_all(dir + "/b.f64");
    std::vector<double> b(rb.size() / 8);
    std::memcpy(b.data(), rb.data(), rb.size());
    auto same = [&](const SkylineMatrix& S, double tol, double atol) {
        CHECK(S.rows() == nrow && S.cols() == ncol && S.get_ia().size() == ia.size());
        for (uint i = 0; i <= nrow; i++) CHECK(S.get_ia()[i] == ia[i]);
        for (uint k = 0; k < nnz; k++) {
            CHECK(S.get_ja()[k] == ja[k]);
            CHECK(std::fabs(S.get_a()[k] - a[k]) <= tol * std::fabs(a[k]) + atol);
        }
    };
    SkylineMatrix S1, S2, S3;
    S1.load(dir + "/ref_A.dat", BINARY, false);
    same(S1, 0.0, 0.0);  // BINARY: the same bits
    S2.load(dir + "/ref_A.crs", ASCII, false);
    same(S2, 1e-15, 0.0);  // 16 significant digits
    S3.load(dir + "/ref_A.mm", MATRIX_MARKET, true);
    same(S3, 1e-15, 5e-16);  // 15 decimals after the point (fixed notation)
    Vector v;
    load(v, dir + "/ref_b.crs", ASCII);
    CHECK(v.size() == b.size());
    for (size_t i = 0; i < b.size(); i++) CHECK(std::fabs(v[i] - b[i]) <= 1e-15 * std::fabs(b[i]));
    Vector w;
    CHECK(throws([&] { load(w, dir + "/ref_b.dat", BINARY); }, "vector.cc:42-46"));
    std::printf("ok\n");
    return 0;
}

static int solve(int argc, char** argv) {
    if (argc != 10) return 2;
    uint nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]);
    SPEMesh mesh(nx, ny, nz, argv[5]);
    Config cfg;
    cfg.prec = MULTI_SPLIT_PREC;
    cfg.prec_conf_file = argv[6];
    cfg.fp32 = std::atoi(argv[8]) != 0;
    double eps = std::atof(argv[7]);
    SkylineMatrix A;
    Vector b;
    mesh.construct_matrix_dirichlet(A, b, 1.0);
    std::unique_ptr<PrecBase> B(make_prec(A, cfg));
    Vector x(A.size());
    SolverStats stats;
    PCGSolver(A, b, *B, x, stats, eps, NORM_L2, true);
    Vector r;
    residual(A, b, x, r);
    dump(argv[9], x, BINARY);
    std::printf("niter %u rel %.6e\n", stats.niter, stats.final_rel);
    return 0;
}

int main(int argc, char** argv) {
    try {
        if (argc >= 3 && std::string(argv[1]) == "cpu") return cpu(argv[2]);
        if (argc >= 2 && std::string(argv[1]) == "solve") return solve(argc, argv);
        if (argc >= 3 && std::string(argv[1]) == "ref-files") return ref_files(argv[2]);
        std::fprintf(stderr, "usage: host_api_test cpu <dir> | solve ...\n");
        return 2;
    } catch (const Exception& e) {
        std::fprintf(stderr, "Exception: %s\n", e.what());
        return 3;
    }
}
