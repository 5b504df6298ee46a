/*
 * C++ host interface of ml_prec_b200, mirroring the ml_prec types and calls on
 * the PCG / multi-split / uh_cheb hot path so that a program written against
 * the reference compiles against this header with its names unchanged:
 *
 *   uvector<T>, Vector                   include/uvector.h:19-194, vector.h:9
 *   CSRMatrix, SkylineMatrix, DumpType   modules/matrix/matrix.h:12-291
 *   SPEMesh                              modules/mesh/mesh.h:52-83, spe.cc
 *   Config, PrecType, SolverType         project/config.h:10-86
 *   ConfigFile                           modules/config_file/config_file.h
 *   PrecBase                             modules/prec/prec_base.h:8-12
 *   MultiSplitPrec(A, cfg)               multi_split_prec.h:105
 *   Prec(A, cfg) (uh_cheb)               cheb_prec.h:115
 *   SolverStats, NormType, PCGSolver     modules/solvers/solvers.h:9-32
 *   generate_x0                          modules/solvers/solvers.cc:9-21
 *   Exception, THROW_EXCEPTION           include/exception.h:24-29
 *
 * Everything numerical runs on the GPU through the C ABI (mlp_b200.h): the
 * matrix keeps a device copy, the preconditioners are device hierarchies, and
 * PCGSolver runs the whole iteration on the device. There is no host
 * computation path: PCGSolver with a preconditioner that is not a device
 * preconditioner throws.
 */
#ifndef ML_PREC_B200_HOST_H
#define ML_PREC_B200_HOST_H

#include <cstdint>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mlp_b200.h"

typedef unsigned int uint;

/* ---- errors (include/exception.h) --------------------------------------- */
class Exception : public std::exception {
    std::string msg_;

public:
    explicit Exception(const std::string& msg) : msg_(msg) {}
    const char* what() const noexcept override { return msg_.c_str(); }
};

#define THROW_EXCEPTION(stream_expr)                                                        \
    do {                                                                                    \
        std::ostringstream mlp_os_;                                                         \
        mlp_os_ << __FILE__ << ":" << __LINE__ << ": " << stream_expr;                      \
        throw Exception(mlp_os_.str());                                                     \
    } while (0)

/* Throws Exception with mlp_last_error() when a C-ABI call fails. */
void mlp_check(int status, const char* what);

/* ---- vectors (uvector.h, vector.h) -------------------------------------- */
template <class T>
class uvector : public std::vector<T> {
public:
    typedef uint size_type;
    uvector() {}
    explicit uvector(size_t n) : std::vector<T>(n) {}
    uvector(size_t n, const T& v) : std::vector<T>(n, v) {}
    uint size() const { return (uint)std::vector<T>::size(); }
};
typedef uvector<double> Vector;

enum DumpType { ASCII, BINARY, HYPRE, MATRIX_MARKET };

void dump(const std::string& filename, const Vector& v, DumpType type);
void load(Vector& v, const std::string& filename, DumpType type);

/* ---- matrices (matrix.h) ------------------------------------------------- */
class CSRMatrix {
protected:
    uint nrow = 0, ncol = 0;
    uvector<uint> ia, ja;
    uvector<double> a;
    mutable mlp_matrix* dev_ = nullptr;  // device copy, made on first use

public:
    CSRMatrix() {}
    CSRMatrix(const CSRMatrix& B);
    CSRMatrix& operator=(const CSRMatrix& B);
    virtual ~CSRMatrix();

    uint rows() const { return nrow; }
    uint cols() const { return ncol; }
    uint size() const;
    uint nnz() const { return (nrow && ncol) ? ia.back() : 0; }
    void set_size(uint r, uint c) { nrow = r; ncol = c; release_device(); }

    /* Non-const accessors may be used to modify the arrays: they drop the
     * device copy, which the next device call rebuilds. */
    uvector<uint>& get_ia() { release_device(); return ia; }
    uvector<uint>& get_ja() { release_device(); return ja; }
    uvector<double>& get_a() { release_device(); return a; }
    const uvector<uint>& get_ia() const { return ia; }
    const uvector<uint>& get_ja() const { return ja; }
    const uvector<double>& get_a() const { return a; }

    double row_sum(uint i) const;
    bool is_symmetric() const;

    /* BINARY (csrmatrix.cc:174-190), ASCII .crs (:191-217) or MatrixMarket
     * (:218-240; a repeated entry keeps its last value, each row's entries in
     * column order). */
    virtual void load(const std::string& filename, DumpType type = BINARY);

    /* The device-resident matrix (uploaded on first use). */
    mlp_matrix* device() const;
    void release_device() const;
    /* Takes ownership of a device matrix and downloads its arrays. */
    void adopt_device(mlp_matrix* m);

    void swap(CSRMatrix& B);

    friend void multiply(const CSRMatrix& A, const Vector& v, Vector& res, char type);
    friend class SPEMesh;
};

/* y = A v on the device (multiply(A, v, res, 'o'), csrmatrix.cc:260-274);
 * only the 'o' (ordinary) product is available. */
void multiply(const CSRMatrix& A, const Vector& v, Vector& res, char type = 'o');
/* r = b - A x (csrmatrix.cc:293-300), product on the device. */
void residual(const CSRMatrix& A, const Vector& b, const Vector& x, Vector& r);
void dump(const std::string& filename, const CSRMatrix& A, DumpType type);

/* CSR with the diagonal first in every row (skyline.cc). */
class SkylineMatrix : public CSRMatrix {
public:
    SkylineMatrix() {}
    using CSRMatrix::load;
    /* transform: move each row's diagonal to the front (skyline.cc:30-58). */
    void load(const std::string& filename, DumpType type, bool transform);
};

/* ---- mesh (mesh.h, spe.cc) ----------------------------------------------- */
class SPEMesh {
    uint nx, ny, nz, N;
    std::vector<double> kx, ky, kz;

public:
    static const uint knx = 60, kny = 220, knz = 85, kN = 60 * 220 * 85;

    /* Reads the permeability blocks (kx, ky, kz; 1,122,000 values each) from
     * "spe_perm.dat" in the working directory, text as in spe.cc:28-41, or
     * from perm_file (text, or raw binary doubles when it ends in ".bin"). */
    SPEMesh(uint nx = 60, uint ny = 220, uint nz = 85, const std::string& perm_file = "spe_perm.dat");
    /* Permeability given directly (each array kN values). */
    SPEMesh(uint nx, uint ny, uint nz, const std::vector<double>& kx, const std::vector<double>& ky,
            const std::vector<double>& kz);

    uint index(uint i, uint j, uint k) const { return k * ny * nx + j * nx + i; }
    uint get_n(char t) const { return t == 'x' ? nx : t == 'y' ? ny : nz; }

    /* construct_matrix(A, c) (spe.cc:69-131), assembled on the device. */
    void construct_matrix(SkylineMatrix& A, double c) const;
    /* The same with p = 1 on the x = 0 face and p = 0 on the x = max face
     * (half-cell transmissibility on the diagonal, the p = 1 term moved to b);
     * the reference matrix has no Dirichlet faces. */
    void construct_matrix_dirichlet(SkylineMatrix& A, Vector& b, double c) const;
};

/* ---- configuration (project/config.h) ------------------------------------ */
enum SolverType { PCG_SOLVER, CHEB_SOLVER, SIMPLE_SOLVER, GMRES_SOLVER, DIRECT_SOLVER };
enum PrecType {
    AMG_PREC, DIAG_PREC, COMP_PREC, GS_PREC, ID_PREC, BGS_PREC, RBGS_PREC,
    SYM_SPLIT_PREC, MULTI_SPLIT_PREC, UH_CHEB_PREC
};

struct Config {
    std::vector<uint> niters;
    std::vector<double> sigmas;
    double c = 1.0;
    uint nx = 60, ny = 220, nz = 85;
    uint ntests = 1;
    bool use_tails = true;
    bool optimize_storage = true;
    bool nonsym_matrix = false;
    double nonsym_shift = 0.1;
    SolverType solver = PCG_SOLVER;
    PrecType prec = UH_CHEB_PREC;
    uint coarse_n = 0;
    uint max_levels = 30;
    bool dump_data = false;
    std::string prec_conf_file;
    std::string dir = "results/";
    std::string matrix;
    std::string vector;
    /* additions of this implementation */
    bool fp32 = false;          // FP32-stored hierarchy inside flexible FP64 PCG
    bool autotune = false;      // time the row kernels' launch shapes at build
    bool dirichlet = false;     // x-face Dirichlet terms of the benchmark problem
    double eps = 1e-6;          // main.cc:129 fixes 1e-6; here it is an option
    std::string perm_file = "spe_perm.dat";

    Config() : niters(1, 2), sigmas(1, 3.0) {}
};
std::ostream& operator<<(std::ostream& os, const Config& cfg);

/* key = value files (config_file.h): '#' comments, values continued on the
 * following lines that hold no delimiter, keys and values trimmed, a later
 * key overrides an earlier one, reading stops at the sentry line. */
class ConfigFile {
    std::string delim_, comment_, sentry_;
    std::map<std::string, std::string> contents_;

    template <class T>
    static T as(const std::string& s);

public:
    struct file_not_found {
        std::string filename;
        explicit file_not_found(const std::string& f = std::string()) : filename(f) {}
    };
    struct key_not_found {
        std::string key;
        explicit key_not_found(const std::string& k = std::string()) : key(k) {}
    };

    ConfigFile() : delim_("="), comment_("#"), sentry_("EndConfigFile") {}
    ConfigFile(const std::string& filename, const std::string& delimiter = "=", const std::string& comment = "#",
               const std::string& sentry = "EndConfigFile");

    void parse(std::istream& is);
    bool keyExists(const std::string& key) const { return contents_.count(key) != 0; }
    template <class T>
    T read(const std::string& key) const {
        auto it = contents_.find(key);
        if (it == contents_.end()) throw key_not_found(key);
        return as<T>(it->second);
    }
    template <class T>
    T read(const std::string& key, const T& value) const {
        auto it = contents_.find(key);
        return it == contents_.end() ? value : as<T>(it->second);
    }
    template <class T>
    bool readInto(T& var, const std::string& key) const {
        auto it = contents_.find(key);
        if (it == contents_.end()) return false;
        var = as<T>(it->second);
        return true;
    }
    template <class T>
    bool readInto(T& var, const std::string& key, const T& value) const {
        bool found = readInto(var, key);
        if (!found) var = value;
        return found;
    }
    template <class T>
    void add(const std::string& key, const T& value) {
        std::ostringstream os;
        os << value;
        contents_[key] = os.str();
    }
    void remove(const std::string& key) { contents_.erase(key); }
};

template <>
inline std::string ConfigFile::as<std::string>(const std::string& s) { return s; }
template <>
inline bool ConfigFile::as<bool>(const std::string& s) {
    std::string t;
    for (char ch : s) t += (char)std::toupper((unsigned char)ch);
    return !(t == "FALSE" || t == "F" || t == "NO" || t == "N" || t == "0" || t == "NONE");
}
template <class T>
inline T ConfigFile::as(const std::string& s) {
    std::istringstream is(s);
    T v{};
    is >> v;
    return v;
}

/* ---- preconditioners ------------------------------------------------------ */
class PrecBase {
public:
    virtual ~PrecBase() {}
    virtual void solve(Vector& f, Vector& x) const = 0;
};

/* A preconditioner whose hierarchy lives on the GPU. */
class DevicePrec : public PrecBase {
protected:
    mlp_prec* h_ = nullptr;
    bool fp32_ = false;
    DevicePrec() {}

public:
    DevicePrec(const DevicePrec&) = delete;
    DevicePrec& operator=(const DevicePrec&) = delete;
    ~DevicePrec() override;
    /* x = B f with host vectors (PrecBase::solve, prec_base.h:11). */
    void solve(Vector& f, Vector& x) const override;
    mlp_prec* handle() const { return h_; }
    bool fp32() const { return fp32_; }
    uint nlevels() const;
    mlp_level_info level_info(uint l) const;
    double setup_seconds() const { return t_setup_; }

protected:
    double t_setup_ = 0;
    void create(const SkylineMatrix& A, const mlp_prec_cfg& c);
};
std::ostream& operator<<(std::ostream& os, const DevicePrec& B);

/* MultiSplitPrec(A, cfg) (multi_split_constr.cc:170-266): parameters from
 * cfg.prec_conf_file (msplit.cfg keys q, inner_iter, level_niter, lu_method,
 * elim_order, elim_stop, degree_max, coarse_n, max_levels; the file overrides
 * the command line), else from cfg.sigmas (q), cfg.niters, cfg.use_tails
 * (original / none ordering), cfg.coarse_n and cfg.max_levels. A config file
 * that does not exist, inner_iter = dynamic and lu_method = ilut are errors
 * (the reference continues with an empty q list in the first case). */
class MultiSplitPrec : public DevicePrec {
public:
    MultiSplitPrec(const SkylineMatrix& A, const Config& cfg);
};

/* Prec (uh_cheb) (cheb_constr.cc:163-248): beta = cfg.sigmas per level,
 * Chebyshev degree = cfg.niters per level, cfg.use_tails. */
class Prec : public DevicePrec {
public:
    Prec(const SkylineMatrix& A, const Config& cfg);
    double lmin() const;
    double lmax() const;
};

/* SymPrec(A, cfg) (sym_prec.h:13-27): the uh_cheb Prec of A's symmetric part
 * (a_ij = max(a_ij, a_ji) off the diagonal), applied as a PCG solve to 1e-14. */
class SymPrec : public DevicePrec {
public:
    SymPrec(const SkylineMatrix& A, const Config& cfg);
};

/* The preconditioner switch of main.cc:100-114 for the kinds this library
 * implements (MULTI_SPLIT_PREC, UH_CHEB_PREC, SYM_SPLIT_PREC); other kinds throw. */
PrecBase* make_prec(const SkylineMatrix& A, const Config& cfg);

/* ---- solver (solvers.h) ---------------------------------------------------- */
enum NormType { NORM_L2, NORM_A, NORM_B_1 };

struct SolverStats {
    double t_resid = 0, t_resid_total = 0;  // not measured separately on the device (0)
    double t_prec = 0, t_prec_total = 0;    // not measured separately on the device (0)
    double t_const = 0;                     // device time of the preconditioner build, when known
    double t_sol = 0;                       // device time of the PCG solve, seconds
    uint niter = 0;
    /* additions of this implementation */
    double init_norm = 0, final_norm = 0, final_rel = 0;
};
std::ostream& operator<<(std::ostream& os, const SolverStats& stats);

/* PCGSolver (pcg.cc:8-102): x0 from generate_x0, stop at ||r|| / ||r0|| <=
 * eps with the 1e-14 absolute floor (solvers.cc:49-58), the whole iteration
 * on the device. B must be a DevicePrec; only NORM_L2 is implemented. An
 * FP32 hierarchy runs the flexible (Polak-Ribiere) iteration. Throws
 * Exception on <Ap, p> <= 0, "No need to iterate", NaN, or the iteration
 * cap (10,000). */
void PCGSolver(const CSRMatrix& A, const Vector& b, const PrecBase& B, Vector& x, SolverStats& stats,
               double eps = 1e-10, NormType norm_type = NORM_L2, bool silent = false);

/* ChebSolver(A, lmin, lmax, b, B, x, eps, norm, silent) (solvers.h:33-34,
 * cheb.cc:9-100) on the device: the Chebyshev iteration with preconditioner B
 * (a device preconditioner; main.cc passes uh_cheb's level-0 lmin / lmax). */
void ChebSolver(const CSRMatrix& A, double lmin, double lmax, const Vector& b, const PrecBase& B, Vector& x,
                double eps = 1e-10, NormType norm_type = NORM_L2, bool silent = false);

void generate_x0(Vector& x);

/* Command-line parsing of main_helper.cc:59-250 for the options of this path
 * (-a -b -c -C -d -D -h -m -M -N -o -O -p -s -t -u -v -x -y -z) plus
 * --eps, --fp32, --dirichlet and --perm. Returns 0 on success. */
int set_params(int argc, char* argv[], Config& cfg);
void construct_matrix(const Config& cfg, const SPEMesh& mesh, SkylineMatrix& A);
void construct_vector(const Config& cfg, Vector& b);
double avg_time(const std::vector<double>& times);

#endif
