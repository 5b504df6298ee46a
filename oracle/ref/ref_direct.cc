// Test-infrastructure shim: the reference's coarsest-level hook DirectSolver
// (multi_split_solve.cc:77-83, declared in solvers.h:40-44) normally calls
// UMFPACK (umfpack.cc:17-56), which is absent here. This shim keeps the hook's
// signature and caching contract (factor once on the first call, keep the factor
// behind the Numeric pointer, solve on every call) and, like UMFPACK, solves the
// coarse system exactly. The multi-split coarse matrix is not symmetric (links are
// dropped one-sidedly), so the reference's dense Cholesky dpotrf (dmatrix.cc:448-478,
// which reads only the upper triangle) does not apply; a dense LU without pivoting
// (right-looking, row-major) is used instead.
#include "modules/solvers/solvers.h"
#include "modules/matrix/matrix.h"

#include <vector>

namespace {
struct DenseLU {
    uint n;
    std::vector<double> a;
};
}

void DirectSolver(const CSRMatrix& A, const Vector& b, Vector& x, void*& Symbolic, void*& Numeric,
                  SolverStats& stats, bool silent) {
    (void)stats; (void)silent;
    if (Numeric == NULL) {
        DenseLU* f = new DenseLU;
        const uint n = A.size();
        f->n = n;
        f->a.assign((size_t)n * n, 0.0);
        const uvector<uint>& ia = A.get_ia();
        const uvector<uint>& ja = A.get_ja();
        const uvector<double>& av = A.get_a();
        for (uint i = 0; i < n; i++)
            for (uint j = ia[i]; j < ia[i + 1]; j++) f->a[(size_t)i * n + ja[j]] = av[j];
        double* a = &f->a[0];
        for (uint k = 0; k < n; k++) {
            double p = a[(size_t)k * n + k];
            if (p == 0.0) THROW_EXCEPTION("zero pivot in the coarse LU at row " << k);
            for (uint i = k + 1; i < n; i++) {
                double l = a[(size_t)i * n + k] / p;
                a[(size_t)i * n + k] = l;
                if (l != 0.0)
                    for (uint j = k + 1; j < n; j++) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
            }
        }
        Numeric = f;
        Symbolic = f;
    }
    DenseLU* f = (DenseLU*)Numeric;
    const uint n = f->n;
    const double* a = &f->a[0];
    for (uint i = 0; i < n; i++) {
        double s = b[i];
        for (uint j = 0; j < i; j++) s -= a[(size_t)i * n + j] * x[j];
        x[i] = s;
    }
    for (int i = (int)n - 1; i >= 0; i--) {
        double s = x[i];
        for (uint j = i + 1; j < n; j++) s -= a[(size_t)i * n + j] * x[j];
        x[i] = s / a[(size_t)i * n + i];
    }
}

void DirectSolver_free(void*& Symbolic, void*& Numeric) {
    delete (DenseLU*)Numeric;
    Numeric = Symbolic = NULL;
}
