// Host destination of a system-matrix build (csr_build.cuh); plain C++.
#pragma once

namespace sgd {

// Host destination of a build.  Either triplets (the reference's spmat: per
// entry three doubles row, column, value; capacity in entries) or CSR
// (rowptr[nrows + 1] int64, cols int32, vals FP64; capacity in entries).
// With no destination the build only counts.
struct CsrOut {
    double* triplets = nullptr;
    long long* rowptr = nullptr;
    int* cols = nullptr;
    double* vals = nullptr;
    long long cap = 0;
    bool counting() const { return !triplets && !rowptr && !cols && !vals; }
};

}  // namespace sgd
