// C++ host interface over the C ABI: matrices, configuration, the
// preconditioner factory and PCGSolver with the reference's signatures.
#include "ml_prec.h"

#include <getopt.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iterator>
#include <memory>
#include <numeric>

void mlp_check(int status, const char* what) {
    if (status == MLP_OK) return;
    std::ostringstream os;
    os << what << ": " << mlp_last_error() << " (status " << status << ")";
    throw Exception(os.str());
}

/* ---- vectors ---------------------------------------------------------------- */

void dump(const std::string& filename, const Vector& v, DumpType type) {
    std::ofstream os(filename.c_str(), type == BINARY ? std::ios::binary : std::ios::out);
    if (!os.good()) THROW_EXCEPTION("Could not open \"" << filename << "\" for write");
    const uint n = v.size();
    if (type == ASCII) {
        os << "# Vector size\n" << n << "\n# Vector values\n" << std::scientific << std::setprecision(15);
        for (uint i = 0; i < n; i++) os << v[i] << "\n";
    } else if (type == HYPRE) {
        os << "0 " << n - 1 << "\n" << std::scientific << std::setprecision(15);
        for (uint i = 0; i < n; i++) os << i << " " << v[i] << "\n";
    } else if (type == BINARY) {
        // size, then all n doubles (vector.cc:42-46 writes only n * 4 bytes of them)
        os.write(reinterpret_cast<const char*>(&n), sizeof(uint));
        os.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)n * sizeof(double));
    } else {
        THROW_EXCEPTION("Not implemented");
    }
}

void load(Vector& v, const std::string& filename, DumpType type) {
    if (type == ASCII) {
        std::ifstream is(filename.c_str());
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << filename << "\"");
        std::string line;
        std::getline(is, line);  // "# Vector size"
        uint n = 0;
        is >> n;
        std::getline(is, line);
        std::getline(is, line);  // "# Vector values"
        v.assign(n, 0.0);
        for (uint i = 0; i < n; i++) is >> v[i];
        if (!is) THROW_EXCEPTION("Short vector file \"" << filename << "\"");
    } else if (type == BINARY) {
        std::ifstream is(filename.c_str(), std::ios::binary | std::ios::ate);
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << filename << "\"");
        const uint64_t bytes = (uint64_t)is.tellg();
        is.seekg(0);
        uint n = 0;
        is.read(reinterpret_cast<char*>(&n), sizeof(uint));
        if (n && bytes == sizeof(uint) + (uint64_t)n * sizeof(uint))
            // the reference's BINARY vector dump writes n * sizeof(uint) bytes of the
            // n doubles (vector.cc:42-46): half of the values are not in the file
            THROW_EXCEPTION("Vector file \"" << filename << "\" holds " << n << " values in " << n * sizeof(uint)
                            << " bytes (the reference's BINARY vector dump, vector.cc:42-46, drops half of "
                               "them); write it as ASCII");
        v.assign(n, 0.0);
        is.read(reinterpret_cast<char*>(v.data()), (std::streamsize)n * sizeof(double));
        if (!is) THROW_EXCEPTION("Short vector file \"" << filename << "\"");
    } else {
        THROW_EXCEPTION("Not implemented");
    }
}

/* ---- matrices ---------------------------------------------------------------- */

CSRMatrix::CSRMatrix(const CSRMatrix& B) : nrow(B.nrow), ncol(B.ncol), ia(B.ia), ja(B.ja), a(B.a) {}

CSRMatrix& CSRMatrix::operator=(const CSRMatrix& B) {
    if (this != &B) {
        release_device();
        nrow = B.nrow;
        ncol = B.ncol;
        ia = B.ia;
        ja = B.ja;
        a = B.a;
    }
    return *this;
}

CSRMatrix::~CSRMatrix() { release_device(); }

uint CSRMatrix::size() const {
    if (nrow != ncol) THROW_EXCEPTION("size was called for rectangular matrix: nrow = " << nrow << ", ncol = " << ncol);
    return nrow;
}

double CSRMatrix::row_sum(uint i) const { return std::accumulate(a.begin() + ia[i], a.begin() + ia[i + 1], 0.0); }

bool CSRMatrix::is_symmetric() const {
    if (nrow != ncol) return false;
    for (uint i = 0; i < nrow; i++)
        for (uint k = ia[i]; k < ia[i + 1]; k++) {
            uint j = ja[k];
            bool found = false;
            for (uint m = ia[j]; m < ia[j + 1]; m++)
                if (ja[m] == i) {
                    found = a[m] == a[k];
                    break;
                }
            if (!found) return false;
        }
    return true;
}

void CSRMatrix::release_device() const {
    if (dev_) {
        mlp_matrix_destroy(dev_);
        dev_ = nullptr;
    }
}

mlp_matrix* CSRMatrix::device() const {
    if (!dev_) {
        if (nrow != ncol) THROW_EXCEPTION("device matrices must be square");
        mlp_check(mlp_matrix_create(nrow, ia.data(), ja.data(), a.data(), &dev_), "mlp_matrix_create");
    }
    return dev_;
}

void CSRMatrix::adopt_device(mlp_matrix* m) {
    release_device();
    uint32_t n = 0, nz = 0;
    mlp_check(mlp_matrix_size(m, &n, &nz), "mlp_matrix_size");
    nrow = ncol = n;
    ia.resize(n + 1);
    ja.resize(nz);
    a.resize(nz);
    mlp_check(mlp_matrix_download(m, ia.data(), ja.data(), a.data()), "mlp_matrix_download");
    dev_ = m;
}

void CSRMatrix::swap(CSRMatrix& B) {
    ia.swap(B.ia);
    ja.swap(B.ja);
    a.swap(B.a);
    std::swap(nrow, B.nrow);
    std::swap(ncol, B.ncol);
    std::swap(dev_, B.dev_);
}

void CSRMatrix::load(const std::string& filename, DumpType type) {
    release_device();
    if (type == BINARY) {
        std::ifstream is(filename.c_str(), std::ios::binary);
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << filename << "\"");
        is.read(reinterpret_cast<char*>(&nrow), sizeof(uint));
        is.read(reinterpret_cast<char*>(&ncol), sizeof(uint));
        ia.resize(nrow + 1);
        is.read(reinterpret_cast<char*>(ia.data()), (std::streamsize)(nrow + 1) * sizeof(uint));
        uint nz = ia[nrow];
        ja.resize(nz);
        a.resize(nz);
        is.read(reinterpret_cast<char*>(ja.data()), (std::streamsize)nz * sizeof(uint));
        is.read(reinterpret_cast<char*>(a.data()), (std::streamsize)nz * sizeof(double));
        if (!is) THROW_EXCEPTION("Short matrix file \"" << filename << "\"");
    } else if (type == ASCII) {
        std::ifstream is(filename.c_str());
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << filename << "\"");
        std::string line;
        uint nz = 0;
        std::getline(is, line);  // "# rows cols nonzeros"
        is >> nrow >> ncol >> nz;
        std::getline(is, line);
        std::getline(is, line);  // "# row_ptr"
        ia.resize(nrow + 1);
        for (uint i = 0; i <= nrow; i++) is >> ia[i];
        std::getline(is, line);
        std::getline(is, line);  // "# col_ind"
        ja.resize(nz);
        for (uint k = 0; k < nz; k++) is >> ja[k];
        std::getline(is, line);
        std::getline(is, line);  // "# value"
        a.resize(nz);
        for (uint k = 0; k < nz; k++) is >> a[k];
        if (!is) THROW_EXCEPTION("Short matrix file \"" << filename << "\"");
    } else if (type == MATRIX_MARKET) {
        std::ifstream is(filename.c_str());
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << filename << "\"");
        // banner, then any '%' comment lines, then "rows cols nonzeros". The
        // reference skips exactly one line after the banner (csrmatrix.cc:221-224),
        // so it cannot read its own dumps (csrmatrix.cc:345-351 writes no comment
        // line); reading past the comment lines accepts both.
        std::string line;
        std::getline(is, line);  // banner
        while (is.peek() == '%') std::getline(is, line);
        uint nz = 0;
        is >> nrow >> ncol >> nz;
        // rows as ordered maps: a repeated (i, j) keeps its last value
        std::vector<std::map<uint, double>> rows(nrow);
        for (uint k = 0; k < nz; k++) {
            uint i, j;
            double v;
            is >> i >> j >> v;
            if (!is || i < 1 || j < 1 || i > nrow || j > ncol) THROW_EXCEPTION("Bad MatrixMarket entry " << k);
            rows[i - 1][j - 1] = v;
        }
        ia.assign(1, 0);
        ja.clear();
        a.clear();
        for (uint i = 0; i < nrow; i++) {
            for (auto& e : rows[i]) {
                ja.push_back(e.first);
                a.push_back(e.second);
            }
            ia.push_back(ja.size());
        }
    } else {
        THROW_EXCEPTION("Loading format HYPRE is not applicable to CSRMatrix");
    }
}

void dump(const std::string& filename, const CSRMatrix& A, DumpType type) {
    const uvector<uint>& ia = A.get_ia();
    const uvector<uint>& ja = A.get_ja();
    const uvector<double>& a = A.get_a();
    uint m = A.rows(), n = A.cols(), nz = ia.back();
    std::ofstream os(filename.c_str(), type == BINARY ? std::ios::binary : std::ios::out);
    if (!os.good()) THROW_EXCEPTION("Could not open \"" << filename << "\" for write");
    if (type == BINARY) {
        os.write(reinterpret_cast<const char*>(&m), sizeof(uint));
        os.write(reinterpret_cast<const char*>(&n), sizeof(uint));
        os.write(reinterpret_cast<const char*>(ia.data()), (std::streamsize)(m + 1) * sizeof(uint));
        os.write(reinterpret_cast<const char*>(ja.data()), (std::streamsize)nz * sizeof(uint));
        os.write(reinterpret_cast<const char*>(a.data()), (std::streamsize)nz * sizeof(double));
    } else if (type == ASCII) {
        os << "# rows cols nonzeros\n" << m << " " << n << " " << nz << "\n# row_ptr\n";
        for (uint i = 0; i <= m; i++) os << ia[i] << "\n";
        os << "# col_ind\n";
        for (uint k = 0; k < nz; k++) os << ja[k] << "\n";
        os << "# value\n" << std::scientific << std::setprecision(15);
        for (uint k = 0; k < nz; k++) os << a[k] << "\n";
    } else if (type == MATRIX_MARKET) {
        os << "%%MatrixMarket matrix coordinate real general\n%\n" << m << " " << n << " " << nz << "\n";
        os << std::scientific << std::setprecision(15);
        for (uint i = 0; i < m; i++)
            for (uint k = ia[i]; k < ia[i + 1]; k++) os << i + 1 << " " << ja[k] + 1 << " " << a[k] << "\n";
    } else {
        os << "0 " << m - 1 << " 0 " << n - 1 << "\n" << std::scientific << std::setprecision(15);
        for (uint i = 0; i < m; i++)
            for (uint k = ia[i]; k < ia[i + 1]; k++) os << i << " " << ja[k] << " " << a[k] << "\n";
    }
}

void SkylineMatrix::load(const std::string& filename, DumpType type, bool transform) {
    CSRMatrix::load(filename, type);
    if (!transform) return;
    for (uint i = 0; i < nrow; i++) {
        uint start = ia[i], end = ia[i + 1], d = end;
        for (uint k = start; k < end; k++)
            if (ja[k] == i) {
                d = k;
                break;
            }
        if (d == end) THROW_EXCEPTION("No diagonal element in row " << i);
        // rotate [start, d] right by one so the diagonal comes first, the others keep their order
        std::rotate(ja.begin() + start, ja.begin() + d, ja.begin() + d + 1);
        std::rotate(a.begin() + start, a.begin() + d, a.begin() + d + 1);
    }
}

void multiply(const CSRMatrix& A, const Vector& v, Vector& res, char type) {
    if (type != 'o') THROW_EXCEPTION("only the ordinary product ('o') is implemented on the device");
    if (v.size() != A.cols()) THROW_EXCEPTION("size mismatch: " << v.size() << " != " << A.cols());
    res.resize(A.rows());
    mlp_check(mlp_spmv_host(A.device(), v.data(), res.data()), "mlp_spmv_host");
}

void residual(const CSRMatrix& A, const Vector& b, const Vector& x, Vector& r) {
    Vector Ax;
    multiply(A, x, Ax);
    r.resize(b.size());
    for (uint i = 0; i < b.size(); i++) r[i] = b[i] - Ax[i];
}

/* ---- mesh ------------------------------------------------------------------ */

SPEMesh::SPEMesh(uint nx_, uint ny_, uint nz_, const std::string& perm_file) : nx(nx_), ny(ny_), nz(nz_) {
    if (!nx || !ny || !nz) THROW_EXCEPTION("Wrong mesh dimensions: " << nx << " x " << ny << " x " << nz);
    N = nx * ny * nz;
    std::vector<double> all;
    all.reserve(3 * (size_t)kN);
    bool binary = perm_file.size() > 4 && perm_file.compare(perm_file.size() - 4, 4, ".bin") == 0;
    if (binary) {
        std::ifstream is(perm_file.c_str(), std::ios::binary);
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << perm_file << "\"");
        all.resize(3 * (size_t)kN);
        is.read(reinterpret_cast<char*>(all.data()), (std::streamsize)all.size() * sizeof(double));
        if (!is) THROW_EXCEPTION("Wrong " << perm_file << " size");
    } else {
        std::ifstream is(perm_file.c_str());
        if (!is.good()) THROW_EXCEPTION("Problem reading file \"" << perm_file << "\"");
        std::copy(std::istream_iterator<double>(is), std::istream_iterator<double>(), std::back_inserter(all));
        if (all.size() != 3 * (size_t)kN) THROW_EXCEPTION("Wrong " << perm_file << " size");
    }
    kx.assign(all.begin(), all.begin() + kN);
    ky.assign(all.begin() + kN, all.begin() + 2 * kN);
    kz.assign(all.begin() + 2 * kN, all.end());
}

SPEMesh::SPEMesh(uint nx_, uint ny_, uint nz_, const std::vector<double>& kx_, const std::vector<double>& ky_,
                 const std::vector<double>& kz_)
    : nx(nx_), ny(ny_), nz(nz_), kx(kx_), ky(ky_), kz(kz_) {
    if (!nx || !ny || !nz) THROW_EXCEPTION("Wrong mesh dimensions: " << nx << " x " << ny << " x " << nz);
    if (kx.size() != kN || ky.size() != kN || kz.size() != kN)
        THROW_EXCEPTION("permeability blocks need " << kN << " values each");
    N = nx * ny * nz;
}

void SPEMesh::construct_matrix(SkylineMatrix& A, double c) const {
    mlp_matrix* m = nullptr;
    mlp_check(mlp_matrix_create_spe(nx, ny, nz, kx.data(), ky.data(), kz.data(), c, 0, &m, nullptr),
              "mlp_matrix_create_spe");
    A.adopt_device(m);
}

void SPEMesh::construct_matrix_dirichlet(SkylineMatrix& A, Vector& b, double c) const {
    mlp_matrix* m = nullptr;
    b.assign(N, 0.0);
    mlp_check(mlp_matrix_create_spe(nx, ny, nz, kx.data(), ky.data(), kz.data(), c, 1, &m, b.data()),
              "mlp_matrix_create_spe");
    A.adopt_device(m);
}

/* ---- configuration ------------------------------------------------------------ */

static void trim(std::string& s) {
    size_t b = s.find_first_not_of(" \t\r\n\f\v");
    if (b == std::string::npos) {
        s.clear();
        return;
    }
    size_t e = s.find_last_not_of(" \t\r\n\f\v");
    s = s.substr(b, e - b + 1);
}

ConfigFile::ConfigFile(const std::string& filename, const std::string& delimiter, const std::string& comment,
                       const std::string& sentry)
    : delim_(delimiter), comment_(comment), sentry_(sentry) {
    std::ifstream in(filename.c_str());
    if (!in) throw file_not_found(filename);
    parse(in);
}

void ConfigFile::parse(std::istream& is) {
    std::vector<std::string> lines;
    for (std::string l; std::getline(is, l);) lines.push_back(l);
    auto strip_comment = [&](const std::string& l) {
        size_t p = l.find(comment_);
        return p == std::string::npos ? l : l.substr(0, p);
    };
    auto has_sentry = [&](const std::string& l) {
        std::string t = l;
        trim(t);
        return !sentry_.empty() && t == sentry_;
    };
    size_t i = 0;
    while (i < lines.size()) {
        std::string line = strip_comment(lines[i++]);
        if (has_sentry(line)) break;
        size_t d = line.find(delim_);
        if (d == std::string::npos) continue;
        std::string key = line.substr(0, d), val = line.substr(d + delim_.size());
        // a value continues on the following non-blank lines that hold no delimiter
        while (i < lines.size()) {
            std::string t = lines[i];
            trim(t);
            if (t.empty()) {
                i++;
                break;
            }
            std::string nxt = strip_comment(lines[i]);
            if (nxt.find(delim_) != std::string::npos || has_sentry(nxt)) break;
            std::string tt = nxt;
            trim(tt);
            if (!tt.empty()) val += "\n";
            val += nxt;
            i++;
        }
        trim(key);
        trim(val);
        contents_[key] = val;
    }
}

std::ostream& operator<<(std::ostream& os, const Config& cfg) {
    os << "Level iterations : ";
    for (uint n : cfg.niters) os << n << " ";
    os << "\nLevel sigmas     : ";
    for (double s : cfg.sigmas) os << s << " ";
    os << "\n";
    if (cfg.matrix.empty()) {
        os << "c                : " << cfg.c << "\n";
        os << "Geometry         : " << cfg.nx << " x " << cfg.ny << " x " << cfg.nz << "\n";
    } else {
        os << "Matrix file      : " << cfg.matrix << "\n";
    }
    os << "Prec             : " << (cfg.prec == MULTI_SPLIT_PREC ? "multi_split" : cfg.prec == UH_CHEB_PREC ? "uh_cheb" : "other")
       << "\n";
    if (!cfg.prec_conf_file.empty()) os << "Prec config file : " << cfg.prec_conf_file << "\n";
    os << "Use tails        : " << (cfg.use_tails ? "true" : "false") << "\n";
    os << "Coarse n         : " << cfg.coarse_n << "\n";
    os << "Max levels       : " << cfg.max_levels << "\n";
    os << "FP32 hierarchy   : " << (cfg.fp32 ? "true" : "false") << "\n";
    return os;
}

/* ---- preconditioners ---------------------------------------------------------- */

DevicePrec::~DevicePrec() {
    if (h_) mlp_prec_destroy(h_);
}

void DevicePrec::create(const SkylineMatrix& A, const mlp_prec_cfg& c) {
    auto t0 = std::chrono::steady_clock::now();
    mlp_check(mlp_prec_create(A.device(), &c, &h_), "mlp_prec_create");
    t_setup_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fp32_ = c.fp32 != 0;
}

void DevicePrec::solve(Vector& f, Vector& x) const {
    uint32_t nl = 0;
    mlp_level_info li;
    mlp_check(mlp_prec_nlevels(h_, &nl), "mlp_prec_nlevels");
    mlp_check(mlp_prec_level_info(h_, 0, &li), "mlp_prec_level_info");
    if (f.size() != li.N) THROW_EXCEPTION("size mismatch: " << f.size() << " != " << li.N);
    x.resize(li.N);
    mlp_check(mlp_prec_apply_host(h_, f.data(), x.data()), "mlp_prec_apply_host");
}

uint DevicePrec::nlevels() const {
    uint32_t n = 0;
    mlp_check(mlp_prec_nlevels(h_, &n), "mlp_prec_nlevels");
    return n;
}

mlp_level_info DevicePrec::level_info(uint l) const {
    mlp_level_info li;
    mlp_check(mlp_prec_level_info(h_, l, &li), "mlp_prec_level_info");
    return li;
}

std::ostream& operator<<(std::ostream& os, const DevicePrec& B) {
    uint nl = B.nlevels();
    os << "Number of levels: " << nl << "\n";
    for (uint l = 0; l < nl; l++) {
        mlp_level_info li = B.level_info(l);
        os << "Level " << l << ": N = " << li.N << ", nnz = " << li.nnz;
        if (li.direct) {
            os << " (direct)\n";
            continue;
        }
        os << ", M = " << li.M << ", Md = " << li.Md << ", n = " << li.n << ", q = " << li.q
           << ", niter = " << li.niter << ", L nnz = " << li.L_nnz << ", U nnz = " << li.U_nnz << "\n";
    }
    return os;
}

template <class T>
static std::vector<T> number_list(const std::string& s) {
    std::istringstream is(s);
    std::vector<T> v;
    double x;
    while (is >> x) v.push_back((T)x);
    return v;
}

MultiSplitPrec::MultiSplitPrec(const SkylineMatrix& A, const Config& cfg) {
    std::vector<double> qs;
    std::vector<uint32_t> niters;
    std::vector<double> epss;  // inner_iter = dynamic
    std::string order_s;
    uint32_t coarse_n, nlevels, degree_max = 3;
    if (!cfg.prec_conf_file.empty()) {
        ConfigFile* f = nullptr;
        try {
            f = new ConfigFile(cfg.prec_conf_file);
        } catch (ConfigFile::file_not_found&) {
            THROW_EXCEPTION("Config file \"" << cfg.prec_conf_file << "\" is absent");
        }
        std::unique_ptr<ConfigFile> keep(f);
        qs = number_list<double>(f->read<std::string>("q", "0.8"));
        std::string inner = f->read<std::string>("inner_iter", "fixed");
        std::string lu = f->read<std::string>("lu_method", "exact");
        order_s = f->read<std::string>("elim_order", "original");
        std::string stop = f->read<std::string>("elim_stop", "degree");
        coarse_n = f->read<uint>("coarse_n", 0);
        nlevels = f->read<uint>("max_levels", 15);
        if (inner == "fixed")
            niters = number_list<uint32_t>(f->read<std::string>("level_niter", "5"));
        else if (inner == "dynamic")
            epss = number_list<double>(f->read<std::string>("level_eps", "1e-2"));
        else
            THROW_EXCEPTION("Unknown inner_iter type: " << inner);
        if (lu == "ilut")
            THROW_EXCEPTION("lu_method = ilut is not implemented");
        else if (lu != "exact")
            THROW_EXCEPTION("Unknown lu type: " << lu);
        if (order_s != "none" && order_s != "original" && order_s != "block" && order_s != "simple_1")
            THROW_EXCEPTION("Unknown elim_order type: " << order_s);
        if (stop == "degree")
            degree_max = f->read<uint>("degree_max", 3);
        else if (stop == "goal")
            degree_max = 0;
        else
            THROW_EXCEPTION("Unknown elim_stop type: " << stop);
    } else {
        qs = cfg.sigmas;
        niters.assign(cfg.niters.begin(), cfg.niters.end());
        order_s = cfg.use_tails ? "original" : "none";
        coarse_n = cfg.coarse_n;
        nlevels = cfg.max_levels;
        for (double q : qs)
            if (q >= 1) THROW_EXCEPTION("All sigmas must be < 1");
    }
    if (qs.empty()) THROW_EXCEPTION("empty q list");
    if (niters.empty()) niters.push_back(5);
    mlp_prec_cfg c;
    std::memset(&c, 0, sizeof(c));
    c.kind = MLP_PREC_MSPLIT;
    c.nq = qs.size();
    c.q = qs.data();
    c.nniter = niters.size();
    c.niter = niters.data();
    c.coarse_n = coarse_n;
    c.max_levels = nlevels;
    c.degree_max = degree_max;
    c.order = order_s == "none" ? MLP_ORDER_NONE : order_s == "original" ? MLP_ORDER_ORIGINAL
              : order_s == "block" ? MLP_ORDER_BLOCK : MLP_ORDER_SIMPLE_1;
    c.use_tails = cfg.use_tails;  // the tail group of elim_order = original
    c.neps = epss.size();
    c.level_eps = epss.empty() ? nullptr : epss.data();
    c.fp32 = cfg.fp32;
    c.autotune = cfg.autotune;
    create(A, c);
}

Prec::Prec(const SkylineMatrix& A, const Config& cfg) {
    if (cfg.sigmas.empty() || cfg.niters.empty()) THROW_EXCEPTION("sigmas and niters must not be empty");
    for (double s : cfg.sigmas)
        if (s <= 1) THROW_EXCEPTION("All sigmas must be > 1");
    std::vector<double> sig = cfg.sigmas;
    std::vector<uint32_t> deg(cfg.niters.begin(), cfg.niters.end());
    mlp_prec_cfg c;
    std::memset(&c, 0, sizeof(c));
    c.kind = MLP_PREC_CHEB;
    c.nsigma = sig.size();
    c.sigma = sig.data();
    c.nncheb = deg.size();
    c.ncheb = deg.data();
    c.use_tails = cfg.use_tails;
    c.max_levels = 30;
    c.fp32 = cfg.fp32;
    c.autotune = cfg.autotune;
    create(A, c);
}

SymPrec::SymPrec(const SkylineMatrix& A, const Config& cfg) {
    if (cfg.sigmas.empty() || cfg.niters.empty()) THROW_EXCEPTION("sigmas and niters must not be empty");
    for (double s : cfg.sigmas)
        if (s <= 1) THROW_EXCEPTION("All sigmas must be > 1");
    std::vector<double> sig = cfg.sigmas;
    std::vector<uint32_t> deg(cfg.niters.begin(), cfg.niters.end());
    mlp_prec_cfg c;
    std::memset(&c, 0, sizeof(c));
    c.kind = MLP_PREC_SYM;
    c.nsigma = sig.size();
    c.sigma = sig.data();
    c.nncheb = deg.size();
    c.ncheb = deg.data();
    c.use_tails = cfg.use_tails;
    c.max_levels = 30;
    c.fp32 = cfg.fp32;
    create(A, c);
}

double Prec::lmin() const { return level_info(0).lmin; }
double Prec::lmax() const { return level_info(0).lmax; }

PrecBase* make_prec(const SkylineMatrix& A, const Config& cfg) {
    switch (cfg.prec) {
        case MULTI_SPLIT_PREC: return new MultiSplitPrec(A, cfg);
        case UH_CHEB_PREC: return new Prec(A, cfg);
        case SYM_SPLIT_PREC: return new SymPrec(A, cfg);
        default: THROW_EXCEPTION("only the multi_split, uh_cheb and sym_split preconditioners are implemented");
    }
}

/* ---- solver ---------------------------------------------------------------- */

void generate_x0(Vector& x) { mlp_check(mlp_generate_x0(x.data(), x.size()), "mlp_generate_x0"); }

void PCGSolver(const CSRMatrix& A, const Vector& b, const PrecBase& B, Vector& x, SolverStats& stats, double eps,
               NormType norm_type, bool silent) {
    const DevicePrec* P = dynamic_cast<const DevicePrec*>(&B);
    if (!P) THROW_EXCEPTION("PCGSolver: the preconditioner has no device implementation");
    if (norm_type != NORM_L2) THROW_EXCEPTION("PCGSolver: only NORM_L2 is implemented");
    if (b.size() != A.size()) THROW_EXCEPTION("Wrong size: " << b.size() << " != " << A.size());
    if (x.size() != A.size()) THROW_EXCEPTION("Wrong size: " << x.size() << " != " << A.size());
    mlp_stats st;
    std::memset(&st, 0, sizeof(st));
    int rc = mlp_pcg(A.device(), b.data(), P->handle(), x.data(), eps, 0, P->fp32() ? 1 : 0, &st);
    if (rc == MLP_ERR_NO_ITER) THROW_EXCEPTION("No need to iterate");
    mlp_check(rc, "PCGSolver");
    stats.t_resid = stats.t_resid_total = stats.t_prec = stats.t_prec_total = 0;
    stats.t_const = 0;
    stats.t_sol = st.t_solve_ms / 1e3;
    stats.niter = st.niter;
    stats.init_norm = st.init_norm;
    stats.final_norm = st.final_norm;
    stats.final_rel = st.final_rel;
    if (!silent)
        std::cout << "#" << stats.niter << ": relative -> " << std::scientific << st.final_rel << "   absolute -> "
                  << st.final_norm << std::defaultfloat << std::endl;
}

void ChebSolver(const CSRMatrix& A, double lmin, double lmax, const Vector& b, const PrecBase& B, Vector& x,
                double eps, NormType norm_type, bool silent) {
    const DevicePrec* P = dynamic_cast<const DevicePrec*>(&B);
    if (!P) THROW_EXCEPTION("ChebSolver: the preconditioner has no device implementation");
    if (norm_type != NORM_L2) THROW_EXCEPTION("ChebSolver: only NORM_L2 is implemented");
    if (b.size() != A.size()) THROW_EXCEPTION("Wrong size: " << b.size() << " != " << A.size());
    if (x.size() != A.size()) THROW_EXCEPTION("Wrong size: " << x.size() << " != " << A.size());
    mlp_stats st;
    std::memset(&st, 0, sizeof(st));
    mlp_check(mlp_cheb_solve(A.device(), b.data(), P->handle(), x.data(), lmin, lmax, eps, 0, &st), "ChebSolver");
    if (!silent)
        std::cout << "#" << st.niter << ": relative -> " << std::scientific << st.final_rel << "   absolute -> "
                  << st.final_norm << std::defaultfloat << std::endl;
}

std::ostream& operator<<(std::ostream& os, const SolverStats& stats) {
    os << std::fixed << std::setprecision(3) << "\n";
    os << "Residual time       :  avg = " << stats.t_resid << "\t total = " << stats.t_resid_total << "\n";
    os << "Prec inversion time :  avg = " << stats.t_prec << "\t total = " << stats.t_prec_total << "\n";
    if (stats.t_const) os << "Time of (possible) construction: " << stats.t_const << "\n";
    os << "Number of iter      : " << stats.niter << "\n";
    os << "Time of solution    : " << stats.t_sol << "\n";
    return os << std::defaultfloat;
}

/* ---- command line (main_helper.cc) -------------------------------------------- */

static void usage() {
    std::cout << "Usage: ml_prec_b200 [options]\n"
                 "  -a|--ntests N                    number of tests to perform\n"
                 "  -b|--niters \"n0 n1 ..\"           iterations (Chebyshev degree) per level\n"
                 "  -c C                             reaction coefficient\n"
                 "  -C|--prec-config-file FILE       config file for the preconditioner (msplit.cfg)\n"
                 "  -d|--dump                        dump matrix and vector and exit\n"
                 "     --dir DIR                     directory for the results\n"
                 "  -h|--help                        this help\n"
                 "  -m|--matrix FILE                 matrix input file (.dat binary, .crs ascii, .mm)\n"
                 "  -M|--max-levels N                maximum number of levels\n"
                 "  -N|--coarse-n N                  direct solve of coarse systems of order <= N\n"
                 "  -o|--solver={pcg|cheb}           outer solver\n"
                 "  -p|--prec={uh_cheb|multi_split|sym_split}  preconditioner\n"
                 "  -s|--sigmas \"s0 s1 ..\"           level sigmas (uh_cheb, > 1) or q (multi_split, < 1)\n"
                 "  -t|--use_tails={yes|no}          tail elimination\n"
                 "  -v|--vector FILE                 right-hand side input file\n"
                 "  -x|--nx N  -y|--ny N  -z|--nz N  SPE mesh dimensions\n"
                 "     --eps E                       PCG relative residual (default 1e-6)\n"
                 "     --fp32                        FP32-stored hierarchy, flexible FP64 PCG\n"
                 "     --dirichlet                   p = 1 / p = 0 on the x faces (right-hand side from them)\n"
                 "     --perm FILE                   permeability file (default spe_perm.dat; .bin = raw doubles)\n"
                 "     --autotune                    time the row kernels' launch shapes at build\n";
}

int set_params(int argc, char* argv[], Config& cfg) {
    enum { OPT_EPS = 1000, OPT_FP32, OPT_DIRICHLET, OPT_PERM, OPT_AUTOTUNE };
    static struct option long_options[] = {
        {"ntests", required_argument, nullptr, 'a'},        {"niters", required_argument, nullptr, 'b'},
        {"c", required_argument, nullptr, 'c'},             {"prec-config-file", required_argument, nullptr, 'C'},
        {"dump", no_argument, nullptr, 'd'},                {"dir", required_argument, nullptr, 'D'},
        {"help", no_argument, nullptr, 'h'},                {"matrix", required_argument, nullptr, 'm'},
        {"max-levels", required_argument, nullptr, 'M'},    {"coarse-n", required_argument, nullptr, 'N'},
        {"optimize-storage", required_argument, nullptr, 'O'}, {"solver", required_argument, nullptr, 'o'},
        {"prec", required_argument, nullptr, 'p'},          {"sigmas", required_argument, nullptr, 's'},
        {"use_tails", required_argument, nullptr, 't'},     {"vector", required_argument, nullptr, 'v'},
        {"nx", required_argument, nullptr, 'x'},            {"ny", required_argument, nullptr, 'y'},
        {"nz", required_argument, nullptr, 'z'},            {"eps", required_argument, nullptr, OPT_EPS},
        {"fp32", no_argument, nullptr, OPT_FP32},           {"dirichlet", no_argument, nullptr, OPT_DIRICHLET},
        {"perm", required_argument, nullptr, OPT_PERM},     {"autotune", no_argument, nullptr, OPT_AUTOTUNE},
        {nullptr, 0, nullptr, 0}};
    optind = 1;
    while (true) {
        int idx = 0;
        int ch = getopt_long(argc, argv, "a:b:c:C:dD:hm:M:N:o:O:p:s:t:v:x:y:z:", long_options, &idx);
        if (ch == -1) break;
        std::string arg = optarg ? optarg : "";
        switch (ch) {
            case 'h': usage(); std::exit(0);
            case 'a': cfg.ntests = (uint)std::atoi(arg.c_str()); break;
            case 'b': cfg.niters = number_list<uint>(arg); break;
            case 's': cfg.sigmas = number_list<double>(arg); break;
            case 'c': cfg.c = std::atof(arg.c_str()); break;
            case 'C': cfg.prec_conf_file = arg; break;
            case 'd': cfg.dump_data = true; break;
            case 'D': cfg.dir = arg; break;
            case 'm': cfg.matrix = arg; break;
            case 'v': cfg.vector = arg; break;
            case 'M': cfg.max_levels = (uint)std::atoi(arg.c_str()); break;
            case 'N': cfg.coarse_n = (uint)std::atoi(arg.c_str()); break;
            case 'x': cfg.nx = (uint)std::atoi(arg.c_str()); break;
            case 'y': cfg.ny = (uint)std::atoi(arg.c_str()); break;
            case 'z': cfg.nz = (uint)std::atoi(arg.c_str()); break;
            case 'O':
                if (arg == "yes") cfg.optimize_storage = true;
                else if (arg == "no") cfg.optimize_storage = false;
                else THROW_EXCEPTION("Unknown optimize-storage option \"" << arg << "\"");
                break;
            case 't':
                if (arg == "yes") cfg.use_tails = true;
                else if (arg == "no") cfg.use_tails = false;
                else THROW_EXCEPTION("Unknown use-tails option \"" << arg << "\"");
                break;
            case 'o':
                if (arg == "pcg") cfg.solver = PCG_SOLVER;
                else if (arg == "cheb") cfg.solver = CHEB_SOLVER;
                else THROW_EXCEPTION("Unknown solver type \"" << arg << "\" (pcg and cheb are implemented)");
                break;
            case 'p':
                if (arg == "uh_cheb") cfg.prec = UH_CHEB_PREC;
                else if (arg == "multi_split") cfg.prec = MULTI_SPLIT_PREC;
                else if (arg == "sym_split") cfg.prec = SYM_SPLIT_PREC;
                else THROW_EXCEPTION("Unknown prec type \"" << arg << "\"");
                break;
            case OPT_EPS: cfg.eps = std::atof(arg.c_str()); break;
            case OPT_FP32: cfg.fp32 = true; break;
            case OPT_DIRICHLET: cfg.dirichlet = true; break;
            case OPT_PERM: cfg.perm_file = arg; break;
            case OPT_AUTOTUNE: cfg.autotune = true; break;
            default: return 1;
        }
    }
    if (cfg.prec == UH_CHEB_PREC || cfg.prec == SYM_SPLIT_PREC)
        for (double s : cfg.sigmas)
            if (s <= 1) THROW_EXCEPTION("All sigmas must be > 1");
    if (cfg.solver == CHEB_SOLVER && cfg.prec != UH_CHEB_PREC)  // main_helper.cc:232-233
        THROW_EXCEPTION("Trying to call Chebyshev solver for not UH Cheb preconditioner");
    if (cfg.prec == MULTI_SPLIT_PREC && cfg.prec_conf_file.empty())
        for (double s : cfg.sigmas)
            if (s >= 1) THROW_EXCEPTION("All sigmas must be < 1");
    return 0;
}

double avg_time(const std::vector<double>& times) {
    if (times.empty()) THROW_EXCEPTION("zero length vector");
    std::vector<double> ts = times;
    std::sort(ts.begin(), ts.end());
    if (ts.size() <= 3) return ts[0];
    // drop the smallest and the two largest (main_helper.cc:252-263)
    return std::accumulate(ts.begin() + 1, ts.end() - 2, 0.0) / (ts.size() - 3);
}

void construct_matrix(const Config& cfg, const SPEMesh& mesh, SkylineMatrix& A) {
    if (!cfg.matrix.empty()) {
        DumpType type = BINARY;
        if (cfg.matrix.find(".crs") != std::string::npos) type = ASCII;
        if (cfg.matrix.find(".mm") != std::string::npos) type = MATRIX_MARKET;
        A.load(cfg.matrix, type, true);
        return;
    }
    mesh.construct_matrix(A, cfg.c);
}

void construct_vector(const Config& cfg, Vector& b) {
    if (cfg.vector.empty()) return;
    DumpType type = cfg.vector.find(".crs") != std::string::npos ? ASCII : BINARY;
    load(b, cfg.vector, type);
}
