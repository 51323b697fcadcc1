// Host-side SDP problem data in the reference's storage model.
//
// Mirrors what the reference builds before its main loop: InputData (b, C,
// A_k as per-block SparseMatrix, sdpa_dataset.h:86-111), the block
// classification of pinpal (sdpa_main.cpp:88-131), the per-block
// constraint index (InputData::initialize_index_SDP,
// sdpa_dataset.cpp:253-343), SparseMatrix::changeToDense
// (sdpa_struct.cpp:458-498) and the formula table
// (Newton::computeFormula_SDP, sdpa_newton.cpp:694-819).
#pragma once

#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "dd.h"

namespace sddd {

// One block of one constraint matrix (SparseMatrix).
struct BlockMat {
    bool dense = false;
    int n = 0;
    std::vector<int> row, col;   // COO in input order (sparse)
    std::vector<dd_t> val;       // COO values (sparse) or n*n column-major (dense)
    int nnz() const { return dense ? n * n : (int)row.size(); }
    int effect = 0;              // NonZeroEffect
};

enum Formula { F1 = 0, F2 = 1, F3 = 2 };

struct Problem {
    int m = 0;
    int nBlock = 0;
    std::vector<int> blockStruct;  // |size|, after sign handling
    std::vector<int> blockType;    // 1 SDP, 3 LP (sdpa_main.cpp:114-131)
    std::vector<int> blockNumber;  // index within its kind
    // LP entries (negative block sizes) are carried as SDP blocks of order 1,
    // appended after the data's SDP blocks: the same problem (a 1 x 1
    // positive semidefinite block is a non-negative scalar, its HKM direction
    // and step length are the LP ones, and every quantity the loop tests is a
    // max-abs norm or a sum over all entries), solved by the ordinary path.
    // Blocks 0 .. nSDPdata-1 are the data's SDP blocks; LP entry t (in
    // blockNumber order) is block nSDPdata + t.
    int nSDP = 0, nLP = 0, nSDPdata = 0;
    std::vector<int> sdpSize;      // SDP block sizes (the LP entries' 1s at the end)
    std::vector<dd_t> b;           // objective of the file (b in SDPA's internal names)
    // C and A[k] by SDP block (C holds -F0 as the reference stores it)
    std::map<int, BlockMat> C;
    std::vector<std::map<int, BlockMat>> A;
    std::string title;
    std::vector<std::string> comments;
    // per SDP block l: constraints k touching it, ascending
    std::vector<std::vector<int>> cons;
    // per SDP block l, per position t in cons[l]: formula
    std::vector<std::vector<int>> formula;
    long nDim() const;
};

// QD 2.3.23 decimal reader (dd_real::read, dd_real.cpp:1198-1259).
int dd_read(const char *s, dd_t *out);

// Reads .dat-s (sparse = true) or .dat text exactly as sdpa_io.cpp does,
// including its tokenizer ("%*[^0-9+-]%[^,} \t\n]").  Throws sddd::Error.
Problem read_problem(const std::string &path, bool sparse);
Problem read_problem_text(const std::string &text, bool sparse);
// In-memory construction from COO triplets in file conventions
// (k = 0 for F0, 1-based block/i/j; F0 is negated into C here).
Problem make_problem(int m, int nblock, const int *blockStruct, const dd_t *b, long nnz, const int *k, const int *blk, const int *i, const int *j,
                     const dd_t *val);

// changeToDense for every matrix, per-block constraint lists, formulas.
void finalize_problem(Problem &p, double kappa);

// An initial point file as IO::read(fpInit, xMat, yVec, zMat, sparse) reads
// it (sdpa_io.cpp:152-283): first the file's x (y = -x), then its X and Y
// matrices (target 1 and 2 in sparse files; the SDP blocks of X, then of Y,
// row by row in dense files) into the internal Z and X, each starting as
// lambda I (Solutions::initialize): a sparse entry sets (i, j) and (j, i); a
// dense file sets only the nonzero entries with i <= j (and their mirror).
// X and Z are block spaces (SDP blocks concatenated, column-major).
void read_init_point_text(const std::string &text, bool sparse, const Problem &P, double lambda, std::vector<dd_t> &X, std::vector<dd_t> &y,
                          std::vector<dd_t> &Z);
void read_init_point(const std::string &path, bool sparse, const Problem &P, double lambda, std::vector<dd_t> &X, std::vector<dd_t> &y,
                     std::vector<dd_t> &Z);

// hi + lo as a decimal string of `digits` significant digits (1..60),
// correctly rounded (half to even) from the exact value: "d.ddd...e+XX",
// "0", "nan", "inf" or "-inf".  The reference prints dd values through QD's
// to_string; this conversion is exact instead, so a point written with 34
// digits reads back (QD's parser, as the initial-point reader) to within a
// few units in the last place of the dd.
std::string dd_to_decimal(dd_t x, int digits);
// The inverse of read_init_point_text: a point (internal X, y, Z, block
// spaces as there) as an initial-point file in the layout that reader takes,
// every number with 34 significant digits.  Dense: the file's x (= -y) on
// the first line, then its X (the internal Z) and its Y (the internal X),
// block by block, row by row.  Sparse: the same x line, then "1 l i j v"
// (internal Z) and "2 l i j v" (internal X) for i <= j, diagonal always.
std::string write_init_point_text(const Problem &P, const std::vector<dd_t> &X, const std::vector<dd_t> &y, const std::vector<dd_t> &Z,
                                  bool sparse);

struct Param {
    int maxIteration = 200;
    double epsilonStar = 1.0e-30, lambdaStar = 1.0e+4, omegaStar = 2.0, lowerBound = -1.0e+5, upperBound = 1.0e+5, betaStar = 0.1, betaBar = 0.3,
           gammaStar = 0.9, epsilonDash = 1.0e-30;
};
// Parameter::setDefaultParameter (sdpa_parts.cpp:136-171); type 0 default,
// 1 unstable-but-fast, 2 stable-but-slow.
Param default_param(int type);
// Parameter::readFile (sdpa_parts.cpp:172-183).
Param read_param(const std::string &path);

} // namespace sddd
