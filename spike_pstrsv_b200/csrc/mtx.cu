// MatrixMarket ingest: coordinate real/integer/double files into 0-based CSR, as
// the reference's matrixMarketToCSR (src/misc.c:109-245) which its profiler driver
// (test/runtime_analysis.c:290-292) uses to load matrices.
//
// Same steps: '%' lines are skipped, "m n nnz" is read, entries are 1-based
// triples; symm 'Y'/'y' mirrors every off-diagonal entry (a real symmetric file
// stores one triangle); entries are sorted by (row, column); uplo 'U' keeps
// row <= column, 'L' row >= column, 'N' everything; the row count reported is the
// column count n, as there.  Deliberate differences: row pointers count entries
// per row (the reference advances one pointer per row change, so an empty row
// shifts every later row), the mirrored count is the real one (the reference
// assumes n diagonal entries), equal (row, column) pairs keep file order, and
// "pattern" files or malformed lines are errors instead of undefined reads.
// Host code only; no GPU is needed.

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "spk_internal.cuh"

namespace {

using spk::set_error;

struct Entry {
    long long row, col, ord;
    double v;
};

template <typename T>
T *alloc64(size_t count) {
    void *p = nullptr;
    if (posix_memalign(&p, 64, std::max<size_t>(count, 1) * sizeof(T)) != 0) return nullptr;
    return (T *)p;
}

int read_mtx(const char *path, char uplo, char symm, double **a, int **ia, int **ja, int *nrows, int *nnz_out) {
    if (!path || !a || !ia || !ja || !nrows) {
        set_error(SPK_ERR_ARG, "null argument");
        return SPK_ERR_ARG;
    }
    uplo = (char)toupper((unsigned char)uplo);
    symm = (char)toupper((unsigned char)symm);
    if ((uplo != 'U' && uplo != 'L' && uplo != 'N') || (symm != 'Y' && symm != 'S' && symm != 'N')) {
        set_error(SPK_ERR_ARG, "uplo must be U, L or N and symm Y, S or N (got %c, %c)", uplo, symm);
        return SPK_ERR_ARG;
    }
    FILE *f = fopen(path, "r");
    if (!f) {
        set_error(SPK_ERR_INPUT, "cannot open %s: %s", path, strerror(errno));
        return SPK_ERR_INPUT;
    }
    char line[4096];
    long long m = 0, n = 0, nz = 0;
    bool header = false, pattern = false;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '%') {
            if (!strncmp(line, "%%MatrixMarket", 14) && strstr(line, "pattern")) pattern = true;
            continue;
        }
        if (sscanf(line, "%lld %lld %lld", &m, &n, &nz) == 3) {
            header = true;
            break;
        }
        if (strspn(line, " \t\r\n") != strlen(line)) break;  // a non-blank line that is not a size line
    }
    if (!header || m <= 0 || n <= 0 || nz < 0 || n > 2147483647ll) {
        fclose(f);
        set_error(SPK_ERR_INPUT, "%s: no valid \"rows columns entries\" line", path);
        return SPK_ERR_INPUT;
    }
    if (pattern) {
        fclose(f);
        set_error(SPK_ERR_INPUT, "%s: pattern matrices carry no values (real, integer or double expected)", path);
        return SPK_ERR_INPUT;
    }
    std::vector<Entry> e;
    e.reserve((size_t)(symm == 'Y' ? 2 * nz : nz));
    long long ord = 0;
    for (long long k = 0; k < nz; k++) {
        long long r, c;
        double v;
        if (!fgets(line, sizeof line, f) || sscanf(line, "%lld %lld %lf", &r, &c, &v) != 3) {
            fclose(f);
            set_error(SPK_ERR_INPUT, "%s: entry %lld of %lld is missing or malformed", path, k + 1, nz);
            return SPK_ERR_INPUT;
        }
        if (r < 1 || r > m || c < 1 || c > n) {
            fclose(f);
            set_error(SPK_ERR_INPUT, "%s: entry %lld (%lld, %lld) outside the %lld x %lld matrix", path, k + 1, r, c, m, n);
            return SPK_ERR_INPUT;
        }
        e.push_back({r - 1, c - 1, ord++, v});
        if (symm == 'Y' && r != c) e.push_back({c - 1, r - 1, ord++, v});
    }
    fclose(f);
    std::stable_sort(e.begin(), e.end(),
                     [](const Entry &x, const Entry &y) { return x.row != y.row ? x.row < y.row : x.col < y.col; });
    std::vector<Entry> keep;
    keep.reserve(e.size());
    for (const Entry &x : e)
        if (uplo == 'N' || (uplo == 'U' && x.row <= x.col) || (uplo == 'L' && x.row >= x.col)) keep.push_back(x);
    if (keep.size() > 2147483647ull) {
        set_error(SPK_ERR_TOO_LARGE, "%s: %zu entries exceed int32 indices", path, keep.size());
        return SPK_ERR_TOO_LARGE;
    }
    // the reference sizes its row pointers by the column count n
    const long long rows = n;
    if (m > n) {
        for (const Entry &x : keep)
            if (x.row >= n) {
                set_error(SPK_ERR_INPUT, "%s: row %lld beyond the %lld rows reported (the column count)", path,
                          x.row + 1, n);
                return SPK_ERR_INPUT;
            }
    }
    int *pia = alloc64<int>((size_t)rows + 1);
    int *pja = alloc64<int>(keep.size());
    double *pa = alloc64<double>(keep.size());
    if (!pia || !pja || !pa) {
        free(pia);
        free(pja);
        free(pa);
        set_error(SPK_ERR_NOMEM, "host allocation failed");
        return SPK_ERR_NOMEM;
    }
    std::vector<long long> cnt((size_t)rows + 1, 0);
    for (const Entry &x : keep) cnt[(size_t)x.row + 1]++;
    pia[0] = 0;
    for (long long r = 0; r < rows; r++) pia[r + 1] = (int)(pia[r] + cnt[(size_t)r + 1]);
    for (size_t k = 0; k < keep.size(); k++) {
        pa[k] = keep[k].v;
        pja[k] = (int)keep[k].col;
    }
    *a = pa;
    *ia = pia;
    *ja = pja;
    *nrows = (int)rows;
    if (nnz_out) *nnz_out = (int)keep.size();
    return SPK_OK;
}

}  // namespace

extern "C" {

int spk_mtx_read(const char *path, char uplo, char symm, double **a, int **ia, int **ja, int *n, int *nnz) {
    return read_mtx(path, uplo, symm, a, ia, ja, n, nnz);
}

void spk_mtx_free(double *a, int *ia, int *ja) {
    free(a);
    free(ia);
    free(ja);
}

void matrixMarketToCSR(const char *filename, double **a, MKL_INT **ia, MKL_INT **ja, int *numRows, const char uplo,
                       const char symm) {
    const int rc = read_mtx(filename, uplo, symm, a, ia, ja, numRows, nullptr);
    if (rc != SPK_OK) {
        fprintf(stderr, "matrixMarketToCSR: %s\n", spk_last_error());
        *a = nullptr;
        *ia = nullptr;
        *ja = nullptr;
        *numRows = 0;
    }
}

// The file's base name without its extension (src/misc.c:254-281: the text
// between the last '/' and the last '.' after it).  Where the reference returns
// NULL (no extension) this returns the whole base name.  malloc'd; free().
char *pathToMatrixName(const char *filepath) {
    if (!filepath) return nullptr;
    const char *base = strrchr(filepath, '/');
    base = base ? base + 1 : filepath;
    const char *dot = strrchr(base, '.');
    const size_t len = dot ? (size_t)(dot - base) : strlen(base);
    char *out = (char *)malloc(len + 1);
    if (!out) return nullptr;
    memcpy(out, base, len);
    out[len] = '\0';
    return out;
}

// str1 followed by str2 in a new malloc'd string (src/misc.c:283-297); a NULL
// argument reads as the empty string.
char *strconcat(const char *str1, const char *str2) {
    const size_t l1 = str1 ? strlen(str1) : 0, l2 = str2 ? strlen(str2) : 0;
    char *out = (char *)malloc(l1 + l2 + 1);
    if (!out) return nullptr;
    if (l1) memcpy(out, str1, l1);
    if (l2) memcpy(out + l1, str2, l2);
    out[l1 + l2] = '\0';
    return out;
}

}  // extern "C"
