// SDPA input reading and problem set-up on the host (see problem.h).
#include "problem.h"

#include <algorithm>
#include <cmath>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <system_error>
#include <thread>

#include "common.cuh"

namespace sddd {

long Problem::nDim() const {
    long s = 0;
    for (int n : sdpSize) s += n;
    return s; // the LP entries are among the blocks
}

// ------------------------------------------------------------ decimal reader
// The value of a decimal string exactly as the reference's dd library reads
// it (QD 2.3.23, dd_real::read and npwr in src/dd_real.cpp; QD is
// Copyright (c) 2003-2009 The Regents of the University of California,
// through Lawrence Berkeley National Laboratory, under a modified BSD
// licence).  Bit-identical input needs its rounding steps: every mantissa
// digit folds in as v*10 (dd times double) then + digit (dd plus double),
// and the decimal exponent scales the result once, by 10^|e| built from
// repeated squaring (multiplications of the "*=" shape, squares of QD's sqr)
// and, for e < 0, one dd division of 1 by it.

// Grammar (QD's): leading blanks; then a sequence of digits, at most one
// '.', one sign before the first digit, and optionally 'e'/'E' followed by
// an integer as sscanf("%d") reads it, which ends the scan; anything else
// is an error (-1).
int dd_read(const char *text, dd_t *out) {
    const char *c = text;
    while (*c == ' ') ++c;
    dd_t mant = dd_zero();
    int ndigits = 0, point_at = -1, exp10 = 0;
    bool negative = false, signed_ = false;
    for (; *c != '\0'; ++c) {
        const char ch = *c;
        if (std::isdigit((unsigned char)ch)) {
            mant = dd_add_d(dd_mul_d(mant, 10.0), (double)(ch - '0'));
            ++ndigits;
            continue;
        }
        if (ch == '.') {
            if (point_at >= 0) return -1;
            point_at = ndigits;
            continue;
        }
        if (ch == '+' || ch == '-') {
            if (signed_ || ndigits > 0) return -1;
            signed_ = true;
            negative = ch == '-';
            continue;
        }
        if (ch == 'e' || ch == 'E') {
            if (std::sscanf(c + 1, "%d", &exp10) != 1) return -1;
            break;
        }
        return -1;
    }
    if (point_at >= 0) exp10 -= ndigits - point_at;
    if (exp10 != 0) mant = dd_muleq(mant, dd_pow10(exp10));
    *out = negative ? dd_neg(mant) : mant;
    return 0;
}

// QD's operator=(const char*) turns an unreadable string into NaN.
static dd_t dd_parse(const char *tok) {
    dd_t v;
    if (dd_read(tok, &v) != 0) {
        double nan = std::nan("");
        return dd_make(nan, nan);
    }
    return v;
}
static dd_t dd_parse(const std::string &tok) { return dd_parse(tok.c_str()); }

// --------------------------------------------------------------- tokenizer
// The fscanf patterns of sdpa_io.cpp over an in-memory copy of the file.
namespace {
struct Scanner {
    const std::string &t;
    size_t p = 0;
    explicit Scanner(const std::string &s) : t(s) {}
    static bool signdigit(char c) { return (c >= '0' && c <= '9') || c == '+' || c == '-'; }
    static bool tokdelim(char c) { return c == ',' || c == '}' || c == ' ' || c == '\t' || c == '\n'; }
    // "%*[^0-9+-]": a non-empty run of other characters (else no match)
    bool skip_nonnum() {
        size_t q = p;
        while (q < t.size() && !signdigit(t[q])) ++q;
        if (q == p || q >= t.size()) {
            p = q;
            return false;
        }
        p = q;
        return true;
    }
    // "%d" after the skip
    bool int_(int &v) {
        while (p < t.size() && std::isspace((unsigned char)t[p])) ++p;
        size_t q = p;
        if (q < t.size() && (t[q] == '+' || t[q] == '-')) ++q;
        size_t d = q;
        long acc = 0; // the digits atoi reads
        while (q < t.size() && t[q] >= '0' && t[q] <= '9') {
            if (acc < (1L << 40)) acc = acc * 10 + (t[q] - '0');
            ++q;
        }
        if (q == d) return false;
        if (acc > 2147483647L) acc = 2147483647L; // out of any index range, as strtol saturates
        v = (int)(t[p] == '-' ? -acc : acc);
        p = q;
        return true;
    }
    bool skip_int(int &v) { return skip_nonnum() && int_(v); }
    // "%*[^0-9+-]%[^,} \t\n]"
    bool skip_token(std::string &tok) {
        size_t b, e;
        if (!skip_token_span(b, e)) return false;
        tok = t.substr(b, e - b);
        return true;
    }
    // the same, giving the token's place in the text
    bool skip_token_span(size_t &b, size_t &e) {
        if (!skip_nonnum()) return false;
        size_t q = p;
        while (q < t.size() && !tokdelim(t[q])) ++q;
        if (q == p) return false;
        b = p;
        e = q;
        p = q;
        return true;
    }
};
} // namespace

static void set_blocks(Problem &P, const std::vector<int> &bs) {
    // pinpal, sdpa_main.cpp:114-131
    P.nBlock = (int)bs.size();
    P.blockStruct.resize(P.nBlock);
    P.blockType.resize(P.nBlock);
    P.blockNumber.resize(P.nBlock);
    for (int i = 0; i < P.nBlock; ++i) {
        int s = bs[i];
        if (s >= 2) {
            P.blockType[i] = 1;
            P.blockNumber[i] = P.nSDP++;
            P.blockStruct[i] = s;
            P.sdpSize.push_back(s);
        } else if (s < 0 || s == 1) {
            P.blockType[i] = 3;
            P.blockStruct[i] = s < 0 ? -s : s;
            P.blockNumber[i] = P.nLP;
            P.nLP += P.blockStruct[i];
        } else {
            throw Error(ERR_IO, "block struct");
        }
    }
    P.nSDPdata = P.nSDP;
    P.sdpSize.insert(P.sdpSize.end(), P.nLP, 1);
    P.nSDP += P.nLP;
}

// SparseLinearSpace::setElement_SDP (sdpa_struct.cpp:1217-1249)
static void add_entry(Problem &P, int k, int l2, int i, int j, dd_t v) {
    if (l2 < 0 || l2 >= P.nBlock) throw Error(ERR_IO, "block index out of range in input data");
    if (P.blockType[l2] == 1) {
        int l = P.blockNumber[l2];
        int n = P.blockStruct[l2];
        if (i < 0 || j < 0 || i >= n || j >= n) throw Error(ERR_IO, "out of range in input data");
        BlockMat &M = (k == 0) ? P.C[l] : P.A[k - 1][l];
        M.n = n;
        M.row.push_back(i);
        M.col.push_back(j);
        M.val.push_back(k == 0 ? dd_neg(v) : v);
        M.effect += (i == j) ? 1 : 2;
    } else {
        // LP entry i of this block: its order-1 block (a later entry for the
        // same place overwrites, as change_to_dense keeps the last value)
        if (i != j) throw Error(ERR_IO, "LP part 3rd element != 4th element");
        if (i < 0 || i >= P.blockStruct[l2]) throw Error(ERR_IO, "out of range in input data");
        const int l = P.nSDPdata + P.blockNumber[l2] + i;
        BlockMat &M = (k == 0) ? P.C[l] : P.A[k - 1][l];
        M.n = 1;
        M.row.push_back(0);
        M.col.push_back(0);
        M.val.push_back(k == 0 ? dd_neg(v) : v);
        M.effect += 1;
    }
}

Problem read_problem_text(const std::string &text, bool sparse) {
    Problem P;
    // IO::read(fpData, fpout, m, str), sdpa_io.cpp:428-438: comment lines
    // start with '*' or '"'; the first other line holds m.
    size_t pos = 0;
    bool have_m = false;
    while (pos < text.size()) {
        size_t eol = text.find('\n', pos);
        if (eol == std::string::npos) eol = text.size();
        std::string line = text.substr(pos, eol - pos);
        pos = std::min(eol + 1, text.size());
        if (!line.empty() && (line[0] == '*' || line[0] == '"')) {
            P.comments.push_back(line);
            continue;
        }
        if (std::sscanf(line.c_str(), "%d", &P.m) != 1) throw Error(ERR_IO, "cannot read mDIM");
        have_m = true;
        break;
    }
    if (!have_m || P.m <= 0) throw Error(ERR_IO, "cannot read mDIM");
    const std::string &rest = text; // scanned from pos on, without a copy
    Scanner sc(rest);
    sc.p = pos;
    int nb = 0;
    if (!sc.int_(nb) || nb <= 0) throw Error(ERR_IO, "cannot read nBLOCK");
    std::vector<int> bs(nb);
    for (int l = 0; l < nb; ++l)
        if (!sc.skip_int(bs[l])) throw Error(ERR_IO, "cannot read bLOCKsTRUCT");
    set_blocks(P, bs);
    P.A.resize(P.m);
    P.b.resize(P.m);
    for (int k = 0; k < P.m; ++k) {
        std::string tok;
        if (!sc.skip_token(tok)) throw Error(ERR_IO, "cannot read the objective vector");
        P.b[k] = dd_parse(tok);
    }
    if (sparse) {
        // IO::setElement, sdpa_io.cpp:653-700: the reference stops at the
        // first entry whose indices or value do not read (sscanf "%lf").
        // Here the entries are located first, their values converted on all
        // host cores (each conversion is the same QD read, independent of
        // the others), then taken in file order with the reference's stop
        // and range checks: the problem is the one the serial loop builds.
        struct Ent {
            int k, l, i, j;
            size_t b, e;
        };
        std::vector<Ent> ents;
        ents.reserve((text.size() - pos) / 24 + 16); // a short entry line is ~ 24 bytes
        while (true) {
            Ent en;
            if (!sc.skip_int(en.k) || !sc.skip_int(en.l) || !sc.skip_int(en.i) || !sc.skip_int(en.j) || !sc.skip_token_span(en.b, en.e)) break;
            ents.push_back(en);
        }
        std::vector<dd_t> vals(ents.size());
        std::vector<char> readable(ents.size());
        std::atomic<bool> failed{false};
        auto convert = [&](size_t lo, size_t hi) noexcept {
            try {
                char buf[64];
                std::string big;
                for (size_t q = lo; q < hi; ++q) {
                    const size_t len = ents[q].e - ents[q].b;
                    const char *tok;
                    if (len < sizeof buf) {
                        std::memcpy(buf, rest.data() + ents[q].b, len);
                        buf[len] = 0;
                        tok = buf;
                    } else {
                        big.assign(rest, ents[q].b, len);
                        tok = big.c_str();
                    }
                    double probe;
                    readable[q] = std::sscanf(tok, "%lf", &probe) > 0;
                    if (readable[q]) vals[q] = dd_parse(tok);
                }
            } catch (...) { // a token too large to copy: report it in the caller's thread
                failed = true;
            }
        };
        const size_t ne = ents.size();
        const unsigned nth = ne < 200000 ? 1u : std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
        if (nth == 1) {
            convert(0, ne);
        } else {
            // a thread that cannot be created leaves its share (and every
            // later one) to the calling thread
            std::vector<std::thread> pool;
            unsigned started = 0;
            try {
                for (; started < nth; ++started) pool.emplace_back(convert, ne * started / nth, ne * (started + 1) / nth);
            } catch (const std::system_error &) {
            }
            if (started < nth) convert(ne * started / nth, ne);
            for (auto &th : pool) th.join();
        }
        if (failed) throw Error(ERR_IO, "input data: out of memory while reading the values");
        for (size_t q = 0; q < ne; ++q) {
            if (!readable[q]) break;
            const Ent &en = ents[q];
            if (en.k < 0 || en.k > P.m) throw Error(ERR_IO, "constraint index out of range in input data");
            add_entry(P, en.k, en.l - 1, en.i - 1, en.j - 1, vals[q]);
        }
    } else {
        // dense: every entry of every block, k = 0..m (sdpa_io.cpp:701-786)
        for (int k = 0; k <= P.m; ++k)
            for (int l2 = 0; l2 < P.nBlock; ++l2) {
                int n = P.blockStruct[l2];
                if (P.blockType[l2] == 1) {
                    for (int i = 0; i < n; ++i)
                        for (int j = 0; j < n; ++j) {
                            std::string tok;
                            if (!sc.skip_token(tok)) throw Error(ERR_IO, "dense data ended early");
                            dd_t v = dd_parse(tok);
                            if (i <= j && !dd_is_zero(v)) add_entry(P, k, l2, i, j, v);
                        }
                } else {
                    for (int j = 0; j < n; ++j) {
                        std::string tok;
                        if (!sc.skip_token(tok)) throw Error(ERR_IO, "dense data ended early");
                        dd_t v = dd_parse(tok);
                        if (!dd_is_zero(v)) add_entry(P, k, l2, j, j, v);
                    }
                }
            }
    }
    return P;
}

// The whole file in one string, read in one go.
static bool slurp(const std::string &path, std::string &out) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.clear();
    char buf[1 << 16];
    size_t n;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        const long len = std::ftell(f);
        if (len > 0) out.reserve((size_t)len);
        std::rewind(f);
    }
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
    std::fclose(f);
    return true;
}

Problem read_problem(const std::string &path, bool sparse) {
    std::string text;
    if (!slurp(path, text)) throw Error(ERR_IO, "Cannot open data file " + path);
    return read_problem_text(text, sparse);
}

void read_init_point_text(const std::string &text, bool sparse, const Problem &P, double lambda, std::vector<dd_t> &X, std::vector<dd_t> &y,
                          std::vector<dd_t> &Z) {
    std::vector<long> off(P.nSDP + 1, 0);
    for (int l = 0; l < P.nSDP; ++l) off[l + 1] = off[l] + (long)P.sdpSize[l] * P.sdpSize[l];
    X.assign(off[P.nSDP], dd_zero());
    Z.assign(off[P.nSDP], dd_zero());
    for (int l = 0; l < P.nSDP; ++l) {
        const int n = P.sdpSize[l];
        for (int i = 0; i < n; ++i) X[off[l] + i + (long)n * i] = Z[off[l] + i + (long)n * i] = dd_from(lambda);
    }
    y.assign(P.m, dd_zero());
    Scanner sc(text);
    std::string tok;
    for (int k = 0; k < P.m; ++k) {
        if (!sc.skip_token(tok)) throw Error(ERR_IO, "initial point: the vector ended early");
        y[k] = dd_neg(dd_parse(tok)); // yVec is opposite sign
    }
    // DenseLinearSpace::setElement_SDP (sdpa_struct.cpp:1564-1577)
    auto set = [&](std::vector<dd_t> &M, int l, int i, int j, dd_t v) {
        if (l < 0 || l >= P.nSDP || i < 0 || j < 0 || i >= P.sdpSize[l] || j >= P.sdpSize[l]) throw Error(ERR_IO, "out of range in input data");
        const int n = P.sdpSize[l];
        M[off[l] + i + (long)n * j] = v;
        M[off[l] + j + (long)n * i] = v;
    };
    if (sparse) {
        int target, l, i, j;
        while (sc.skip_int(target) && sc.skip_int(l) && sc.skip_int(i) && sc.skip_int(j) && sc.skip_token(tok)) {
            double probe;
            if (std::sscanf(tok.c_str(), "%lf", &probe) <= 0) break;
            const dd_t v = dd_parse(tok);
            if (l <= P.nSDPdata) {
                set(target == 1 ? Z : X, l - 1, i - 1, j - 1, v);
            } else { // the LP part: entry i (setElement_LP)
                if (i != j) throw Error(ERR_IO, "initial point: LP part 3rd element != 4th element");
                if (i < 1 || i > P.nLP) throw Error(ERR_IO, "out of range in input data");
                set(target == 1 ? Z : X, P.nSDPdata + i - 1, 0, 0, v);
            }
        }
    } else {
        for (int pass = 0; pass < 2; ++pass) { // Z (the file's X), then X (its Y)
            std::vector<dd_t> &M = pass == 0 ? Z : X;
            for (int l = 0; l < P.nSDPdata; ++l) {
                const int n = P.sdpSize[l];
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j) {
                        if (!sc.skip_token(tok)) throw Error(ERR_IO, "initial point: the matrices ended early");
                        const dd_t v = dd_parse(tok);
                        if (i <= j && !dd_is_zero(v)) set(M, l, i, j, v);
                    }
            }
            for (int t = 0; t < P.nLP; ++t) { // then the LP part, nonzero entries
                if (!sc.skip_token(tok)) throw Error(ERR_IO, "initial point: the LP part ended early");
                const dd_t v = dd_parse(tok);
                if (!dd_is_zero(v)) set(M, P.nSDPdata + t, 0, 0, v);
            }
        }
    }
}

void read_init_point(const std::string &path, bool sparse, const Problem &P, double lambda, std::vector<dd_t> &X, std::vector<dd_t> &y,
                     std::vector<dd_t> &Z) {
    std::string text;
    if (!slurp(path, text)) throw Error(ERR_IO, "Cannot open init file " + path);
    read_init_point_text(text, sparse, P, lambda, X, y, Z);
}

// ------------------------------------------------------ exact dd printing
namespace {
// Non-negative integer in base 2^32, least significant limb first.
struct BigNat {
    std::vector<uint32_t> d;
    bool zero() const { return d.empty(); }
    void trim() {
        while (!d.empty() && d.back() == 0) d.pop_back();
    }
    void mul_small(uint32_t f) {
        uint64_t carry = 0;
        for (uint32_t &w : d) {
            const uint64_t t = (uint64_t)w * f + carry;
            w = (uint32_t)t;
            carry = t >> 32;
        }
        if (carry) d.push_back((uint32_t)carry);
    }
    void shl(int k) { // *= 2^k
        while (k >= 31) {
            mul_small(1u << 31);
            k -= 31;
        }
        if (k > 0) mul_small(1u << k);
    }
    uint32_t div_small(uint32_t q) { // /= q, returns the remainder
        uint64_t r = 0;
        for (size_t i = d.size(); i-- > 0;) {
            const uint64_t t = (r << 32) | d[i];
            d[i] = (uint32_t)(t / q);
            r = t % q;
        }
        trim();
        return (uint32_t)r;
    }
    static BigNat from(uint64_t v) {
        BigNat b;
        while (v) {
            b.d.push_back((uint32_t)v);
            v >>= 32;
        }
        return b;
    }
    // a - b for a >= b
    static BigNat sub(const BigNat &a, const BigNat &b) {
        BigNat r = a;
        int64_t borrow = 0;
        for (size_t i = 0; i < r.d.size(); ++i) {
            int64_t t = (int64_t)r.d[i] - borrow - (i < b.d.size() ? (int64_t)b.d[i] : 0);
            borrow = t < 0;
            r.d[i] = (uint32_t)(t + (borrow ? (int64_t)1 << 32 : 0));
        }
        r.trim();
        return r;
    }
    static BigNat add(const BigNat &a, const BigNat &b) {
        BigNat r;
        uint64_t carry = 0;
        for (size_t i = 0; i < std::max(a.d.size(), b.d.size()); ++i) {
            const uint64_t t = (uint64_t)(i < a.d.size() ? a.d[i] : 0) + (i < b.d.size() ? b.d[i] : 0) + carry;
            r.d.push_back((uint32_t)t);
            carry = t >> 32;
        }
        if (carry) r.d.push_back((uint32_t)carry);
        return r;
    }
    std::string decimal() const {
        if (d.empty()) return "0";
        BigNat t = *this;
        std::string out;
        while (!t.zero()) {
            uint32_t r = t.div_small(1000000000u);
            for (int k = 0; k < 9; ++k) {
                out.push_back((char)('0' + r % 10));
                r /= 10;
            }
        }
        while (out.size() > 1 && out.back() == '0') out.pop_back();
        std::reverse(out.begin(), out.end());
        return out;
    }
};
} // namespace

std::string dd_to_decimal(dd_t x, int digits) {
    digits = std::max(1, std::min(60, digits));
    if (std::isnan(x.hi) || std::isnan(x.lo)) return "nan";
    if (std::isinf(x.hi)) return x.hi > 0 ? "inf" : "-inf";
    if (x.hi == 0.0 && x.lo == 0.0) return "0";
    // |x| = |hi| + s |lo| exactly, s = +-1 (|lo| < |hi|); each part an
    // integer significand times a power of two
    const bool neg = x.hi < 0.0 || (x.hi == 0.0 && x.lo < 0.0);
    const double h = std::fabs(x.hi), l = std::fabs(x.lo);
    const bool same = x.hi == 0.0 || x.lo == 0.0 || ((x.hi < 0.0) == (x.lo < 0.0));
    int eh = 0, el = 0;
    const uint64_t mh = h > 0.0 ? (uint64_t)std::ldexp(std::frexp(h, &eh), 53) : 0;
    const uint64_t ml = l > 0.0 ? (uint64_t)std::ldexp(std::frexp(l, &el), 53) : 0;
    eh -= 53;
    el -= 53;
    const int e = h > 0.0 && l > 0.0 ? std::min(eh, el) : (h > 0.0 ? eh : el);
    BigNat A = BigNat::from(mh), B = BigNat::from(ml);
    if (h > 0.0) A.shl(eh - e);
    if (l > 0.0) B.shl(el - e);
    BigNat N = same ? BigNat::add(A, B) : BigNat::sub(A, B);
    // |x| = N 2^e: for e < 0 it is N 5^-e 10^e, an integer times a power of ten
    int dexp = 0;
    if (e >= 0) {
        N.shl(e);
    } else {
        for (int k = 0; k < -e; ++k) N.mul_small(5);
        dexp = e;
    }
    std::string s = N.decimal();
    // round half to even at `digits` significant digits
    if ((int)s.size() > digits) {
        const char next = s[digits];
        bool rest = false;
        for (size_t k = digits + 1; k < s.size(); ++k) rest |= s[k] != '0';
        const bool up = next > '5' || (next == '5' && (rest || ((s[digits - 1] - '0') & 1)));
        dexp += (int)s.size() - digits;
        s.resize(digits);
        if (up) {
            int k = digits - 1;
            while (k >= 0 && s[k] == '9') s[k--] = '0';
            if (k >= 0) {
                s[k]++;
            } else {
                s.insert(s.begin(), '1');
                s.pop_back();
                dexp += 1;
            }
        }
    }
    const int exp10 = dexp + (int)s.size() - 1; // of the first digit
    std::string out = neg ? "-" : "";
    out += s[0];
    if (s.size() > 1) {
        out += '.';
        out.append(s, 1, std::string::npos);
    }
    char eb[16];
    std::snprintf(eb, sizeof eb, "e%+03d", exp10);
    return out + eb;
}

std::string write_init_point_text(const Problem &P, const std::vector<dd_t> &X, const std::vector<dd_t> &y, const std::vector<dd_t> &Z,
                                  bool sparse) {
    std::vector<long> off(P.nSDP + 1, 0);
    for (int l = 0; l < P.nSDP; ++l) off[l + 1] = off[l] + (long)P.sdpSize[l] * P.sdpSize[l];
    if ((long)X.size() < off[P.nSDP] || (long)Z.size() < off[P.nSDP] || (int)y.size() < P.m) throw Error(ERR_ARG, "initial point: arrays too short");
    constexpr int D = 34;
    std::string out = "{";
    for (int k = 0; k < P.m; ++k) {
        if (k) out += ',';
        out += dd_to_decimal(dd_neg(y[k]), D); // the file's x is -y
    }
    out += "}\n";
    if (sparse) {
        for (int pass = 0; pass < 2; ++pass) { // target 1: internal Z (the file's X); 2: internal X (its Y)
            const std::vector<dd_t> &M = pass == 0 ? Z : X;
            for (int t = 0; t < P.nLP; ++t) // the LP part: "target block i i v", block past the SDP ones
                out += std::to_string(pass + 1) + ' ' + std::to_string(P.nSDPdata + 1) + ' ' + std::to_string(t + 1) + ' ' + std::to_string(t + 1) + ' ' +
                       dd_to_decimal(M[off[P.nSDPdata + t]], D) + '\n';
            for (int l = 0; l < P.nSDPdata; ++l) {
                const int n = P.sdpSize[l];
                for (int i = 0; i < n; ++i)
                    for (int j = i; j < n; ++j) {
                        const dd_t v = M[off[l] + i + (long)n * j];
                        if (i != j && dd_is_zero(v)) continue;
                        out += std::to_string(pass + 1) + ' ' + std::to_string(l + 1) + ' ' + std::to_string(i + 1) + ' ' + std::to_string(j + 1) + ' ' +
                               dd_to_decimal(v, D) + '\n';
                    }
            }
        }
    } else {
        for (int pass = 0; pass < 2; ++pass) {
            const std::vector<dd_t> &M = pass == 0 ? Z : X;
            for (int l = 0; l < P.nSDPdata; ++l) {
                const int n = P.sdpSize[l];
                out += "{ ";
                for (int i = 0; i < n; ++i) {
                    out += '{';
                    for (int j = 0; j < n; ++j) {
                        if (j) out += ',';
                        // the reader takes entries with i <= j: write the upper triangle's
                        // values in both places, so the file is symmetric
                        out += dd_to_decimal(M[off[l] + std::min(i, j) + (long)n * std::max(i, j)], D);
                    }
                    out += i + 1 < n ? "}," : "}";
                }
                out += " }\n";
            }
            if (P.nLP > 0) { // the LP part, one list
                out += '{';
                for (int t = 0; t < P.nLP; ++t) {
                    if (t) out += ',';
                    out += dd_to_decimal(M[off[P.nSDPdata + t]], D);
                }
                out += "}\n";
            }
        }
    }
    return out;
}

Problem make_problem(int m, int nblock, const int *blockStruct, const dd_t *b, long nnz, const int *k, const int *blk, const int *i, const int *j,
                     const dd_t *val) {
    if (m <= 0 || nblock <= 0) throw Error(ERR_ARG, "m and nblock must be positive");
    Problem P;
    P.m = m;
    set_blocks(P, std::vector<int>(blockStruct, blockStruct + nblock));
    P.A.resize(m);
    P.b.assign(b, b + m);
    for (long e = 0; e < nnz; ++e) {
        if (k[e] < 0 || k[e] > m) throw Error(ERR_ARG, "constraint index out of range");
        add_entry(P, k[e], blk[e] - 1, i[e] - 1, j[e] - 1, val[e]);
    }
    return P;
}

// SparseMatrix::changeToDense (sdpa_struct.cpp:458-498): at least 20% of the
// n*n entries stored -> dense, later entries overwrite earlier ones.
static void change_to_dense(BlockMat &M) {
    if (M.dense) return;
    const int n = M.n;
    if ((double)M.row.size() < (double)(n * n) * 0.20) return;
    std::vector<dd_t> D((size_t)n * n, dd_zero());
    for (size_t e = 0; e < M.row.size(); ++e) {
        int i = M.row[e], j = M.col[e];
        D[i + (size_t)n * j] = M.val[e];
        D[j + (size_t)n * i] = M.val[e];
    }
    M.dense = true;
    M.val.swap(D);
    M.row.clear();
    M.col.clear();
    M.effect = n * n;
}

void finalize_problem(Problem &P, double kappa) {
    for (auto &kv : P.C) change_to_dense(kv.second);
    for (auto &Ak : P.A)
        for (auto &kv : Ak) change_to_dense(kv.second);
    P.cons.assign(P.nSDP, {});
    for (int k = 0; k < P.m; ++k)
        for (auto &kv : P.A[k]) P.cons[kv.first].push_back(k);
    // formula choice with the reference's dd cost model
    P.formula.assign(P.nSDP, {});
    const dd_t K = dd_from(kappa);
    for (int l = 0; l < P.nSDP; ++l) {
        const auto &cl = P.cons[l];
        const int nc = (int)cl.size();
        std::vector<int> eff(nc);
        for (int t = 0; t < nc; ++t) eff[t] = P.A[cl[t]].at(l).effect;
        // "up": sum of the effects that sort below this one
        std::vector<int> order(nc);
        for (int t = 0; t < nc; ++t) order[t] = t;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return eff[a] != eff[b] ? eff[a] < eff[b] : cl[a] < cl[b]; });
        std::vector<long> up(nc);
        long run = 0;
        for (int s = 0; s < nc; ++s) {
            int t = order[s];
            up[t] = eff[t] + run; // itself plus every (jnz < inz) or (jnz == inz and j < i)
            run += eff[t];
        }
        P.formula[l].resize(nc);
        const dd_t nn = dd_from((double)P.sdpSize[l]);
        for (int t = 0; t < nc; ++t) {
            const BlockMat &M = P.A[cl[t]].at(l);
            dd_t inz = dd_from((double)eff[t]), u = dd_from((double)up[t]);
            dd_t f1 = dd_add(dd_add(dd_mul(dd_mul(K, nn), inz), dd_mul(dd_mul(nn, nn), nn)), dd_mul(K, u));
            dd_t f2 = dd_add(dd_mul(dd_mul(K, nn), inz), dd_mul(dd_mul(K, dd_add_d(nn, 1.0)), u));
            dd_t f3 = dd_div(dd_mul(dd_mul(K, dd_add_d(dd_mul(dd_mul_d(K, 2.0), inz), 1.0)), u), K);
            int f;
            if (M.dense)
                f = dd_lt(f1, f2) ? F1 : F2;
            else if (dd_lt(f1, f2) && dd_lt(f1, f3))
                f = F1;
            else if (dd_lt(f2, f3))
                f = F2;
            else
                f = F3;
            P.formula[l][t] = f;
        }
    }
}

// ---------------------------------------------------------------- params
Param default_param(int type) {
    Param p;
    if (type == 2) { // PARAMETER_STABLE_BUT_SLOW
        p.maxIteration = 1000;
        p.lambdaStar = 1.0e+2;
        p.betaStar = 0.2;
        p.betaBar = 0.4;
        p.gammaStar = 0.5;
    } else if (type == 1) { // PARAMETER_UNSTABLE_BUT_FAST
        p.maxIteration = 100;
        p.lambdaStar = 1.0e+2;
        p.betaStar = 0.01;
        p.betaBar = 0.02;
        p.gammaStar = 0.98;
    }
    return p;
}

Param read_param(const std::string &path) {
    FILE *f = std::fopen(path.c_str(), "r");
    if (!f) throw Error(ERR_IO, "Cannot open parameter file " + path);
    Param p;
    // fscanf("%d%*[^\n]") / fscanf("%lf%*[^\n]") per line
    int rc = std::fscanf(f, "%d%*[^\n]", &p.maxIteration);
    double *dst[] = {&p.epsilonStar, &p.lambdaStar, &p.omegaStar, &p.lowerBound, &p.upperBound, &p.betaStar, &p.betaBar, &p.gammaStar, &p.epsilonDash};
    for (double *d : dst) rc = std::fscanf(f, "%lf%*[^\n]", d);
    (void)rc;
    std::fclose(f);
    return p;
}

} // namespace sddd
