// MT19937 with its state open and a jump-ahead by polynomial arithmetic over
// GF(2); see include/mgbrain/mt19937.h for the method and its sources.
#include "mgbrain/mt19937.h"

#include <mutex>
#include <stdexcept>

namespace MGBrain {

namespace {

constexpr int kM = 397;
constexpr uint32_t kMatrixA = 0x9908b0dfu;
constexpr uint32_t kUpper = 0x80000000u, kLower = 0x7fffffffu;
constexpr int kDegree = 19937;                 // degree of phi (the state's dimension)
constexpr int kWords = (kDegree + 63) / 64 + 1;  // one polynomial below phi's degree, with a spare word

using Poly = std::vector<uint64_t>;

inline bool bit(const Poly& p, size_t i) { return (p[i >> 6] >> (i & 63)) & 1u; }
inline void flip(Poly& p, size_t i) { p[i >> 6] ^= uint64_t(1) << (i & 63); }

// 64 bits of a starting at bit position `pos` (bits past the end read 0).
inline uint64_t bits_at(const Poly& a, size_t pos)
{
    const size_t w = pos >> 6, s = pos & 63;
    uint64_t lo = w < a.size() ? a[w] : 0;
    if (s == 0) return lo;
    const uint64_t hi = w + 1 < a.size() ? a[w + 1] : 0;
    return (lo >> s) | (hi << (64 - s));
}

// c ^= b << m (b and c with enough words for the result)
void xor_shifted(Poly& c, const Poly& b, size_t m, size_t b_bits)
{
    const size_t ws = m >> 6, s = m & 63;
    const size_t nb = (b_bits + 63) / 64;
    for (size_t w = 0; w < nb; ++w) {
        const uint64_t v = b[w];
        if (!v) continue;
        if (w + ws < c.size()) c[w + ws] ^= v << s;
        if (s && w + ws + 1 < c.size()) c[w + ws + 1] ^= v >> (64 - s);
    }
}

// Berlekamp-Massey over GF(2): the connection polynomial C (C[0] = 1,
// s[n] = sum_{i=1..L} C[i] s[n-i]) of the bit sequence s, and its length L.
Poly berlekamp_massey(const std::vector<uint8_t>& s, int& L_out)
{
    const size_t n_bits = s.size();
    const size_t words = n_bits / 64 + 2;
    // r: s reversed, so that sum_i C[i] s[n-i] is C AND a window of r
    Poly r(words, 0);
    for (size_t j = 0; j < n_bits; ++j)
        if (s[n_bits - 1 - j]) flip(r, j);
    Poly C(words, 0), B(words, 0), T;
    C[0] = B[0] = 1;
    size_t L = 0, m = 1;
    for (size_t n = 0; n < n_bits; ++n) {
        // d = sum_{i=0..L} C[i] s[n-i] = parity(C[0..L] & r[N-1-n ...])
        const size_t off = n_bits - 1 - n;
        uint64_t acc = 0;
        const size_t nw = L / 64 + 1;
        for (size_t w = 0; w < nw; ++w) {
            uint64_t cw = C[w];
            if (w == L / 64) cw &= (L % 64 == 63) ? ~uint64_t(0) : ((uint64_t(1) << (L % 64 + 1)) - 1);
            acc ^= cw & bits_at(r, off + 64 * w);
        }
        const bool d = __builtin_parityll(acc);
        if (!d) {
            ++m;
        } else if (2 * L <= n) {
            T = C;
            xor_shifted(C, B, m, n + 1);
            L = n + 1 - L;
            B = T;
            m = 1;
        } else {
            xor_shifted(C, B, m, n + 1);
            ++m;
        }
    }
    L_out = (int)L;
    C.resize(L / 64 + 1);
    return C;
}

struct Phi {
    Poly p;                      // phi, bits 0..kDegree (x^kDegree set)
    std::vector<Poly> shifted;   // phi << b for b = 0..63
};

const Phi& phi()
{
    static Phi f;
    static std::once_flag once;
    std::call_once(once, [] {
        Mt19937 g(1u);
        std::vector<uint8_t> s(2 * kDegree + 64);
        for (auto& b : s) b = g() & 1u;
        int L = 0;
        const Poly C = berlekamp_massey(s, L);
        if (L != kDegree) throw std::runtime_error("MT19937: characteristic polynomial of unexpected degree");
        // phi(x) = x^L C(1/x): coefficient of x^(L-i) is C[i]
        f.p.assign(kWords + 1, 0);
        for (int i = 0; i <= L; ++i)
            if (bit(C, (size_t)i)) flip(f.p, (size_t)(L - i));
        f.shifted.assign(64, Poly(kWords + 2, 0));
        for (int b = 0; b < 64; ++b) xor_shifted(f.shifted[b], f.p, (size_t)b, kDegree + 1);
    });
    return f;
}

// a mod phi, for a of degree < 2 * kDegree (a has 2 * kWords words)
void reduce(Poly& a)
{
    const Phi& f = phi();
    for (long p = (long)a.size() * 64 - 1; p >= kDegree; --p) {
        if (!bit(a, (size_t)p)) continue;
        const size_t sh = (size_t)(p - kDegree);
        const Poly& q = f.shifted[sh & 63];
        const size_t ws = sh >> 6;
        for (size_t w = 0; w < q.size() && w + ws < a.size(); ++w) a[w + ws] ^= q[w];
    }
    a.resize(kWords);
}

// a^2 over GF(2): bit i -> bit 2i
Poly square(const Poly& a)
{
    static uint16_t spread[256];
    static std::once_flag once;
    std::call_once(once, [] {
        for (int v = 0; v < 256; ++v) {
            uint16_t r = 0;
            for (int k = 0; k < 8; ++k)
                if (v >> k & 1) r |= (uint16_t)(1u << (2 * k));
            spread[v] = r;
        }
    });
    Poly r(2 * a.size(), 0);
    for (size_t w = 0; w < a.size(); ++w) {
        const uint64_t v = a[w];
        uint64_t lo = 0, hi = 0;
        for (int k = 0; k < 4; ++k) {
            lo |= (uint64_t)spread[(v >> (8 * k)) & 0xff] << (16 * k);
            hi |= (uint64_t)spread[(v >> (32 + 8 * k)) & 0xff] << (16 * k);
        }
        r[2 * w] = lo;
        r[2 * w + 1] = hi;
    }
    return r;
}

}  // namespace

void Mt19937::seed_with(uint32_t seed)
{
    x_[0] = seed;
    for (int k = 1; k < N; ++k) x_[k] = 1812433253u * (x_[k - 1] ^ (x_[k - 1] >> 30)) + (uint32_t)k;
    i_ = 0;
}

void Mt19937::twist_block()
{
    auto next = [](uint32_t a, uint32_t b, uint32_t c) {
        const uint32_t y = (a & kUpper) | (b & kLower);
        return c ^ (y >> 1) ^ ((y & 1u) ? kMatrixA : 0u);
    };
    int j = 0;
    for (; j < N - kM; ++j) x_[j] = next(x_[j], x_[j + 1], x_[j + kM]);
    for (; j < N - 1; ++j) x_[j] = next(x_[j], x_[j + 1], x_[j + kM - N]);
    x_[N - 1] = next(x_[N - 1], x_[0], x_[kM - 1]);
}

void Mt19937::generate(uint32_t* out, size_t n)
{
    size_t k = 0;
    for (; k < n && i_ != 0; ++k) out[k] = (*this)();
    for (; n - k >= (size_t)N; k += N) {
        twist_block();
        for (int j = 0; j < N; ++j) out[k + j] = temper(x_[j]);
    }
    for (; k < n; ++k) out[k] = (*this)();
}

void Mt19937::discard(uint64_t n)
{
    uint64_t k = 0;
    for (; k < n && i_ != 0; ++k) step();
    for (; n - k >= (uint64_t)N; k += N) twist_block();
    for (; k < n; ++k) step();
}

void Mt19937::add(const Mt19937& o)
{
    for (int k = 0; k < N; ++k) {
        int a = i_ + k, b = o.i_ + k;
        if (a >= N) a -= N;
        if (b >= N) b -= N;
        x_[a] ^= o.x_[b];
    }
}

void Mt19937::clear()
{
    for (int k = 0; k < N; ++k) x_[k] = 0;
}

void Mt19937::state_words(uint32_t* out) const
{
    for (int k = 0; k < N; ++k) out[k] = x_[(i_ + k) % N];
}

void Mt19937::set_state_words(const uint32_t* in)
{
    for (int k = 0; k < N; ++k) x_[k] = in[k];
    i_ = 0;
}

MtJump::MtJump(uint64_t steps) : steps_(steps)
{
    // x^steps mod phi by squaring and multiplying by x, from the top bit
    poly_.assign(kWords, 0);
    poly_[0] = 1;
    int top = 63;
    while (top >= 0 && !((steps >> top) & 1u)) --top;
    for (int b = top; b >= 0; --b) {
        Poly sq = square(poly_);
        reduce(sq);
        poly_ = sq;
        if ((steps >> b) & 1u) {
            // multiply by x: shift left one bit, then reduce the top bit
            uint64_t carry = 0;
            for (auto& w : poly_) {
                const uint64_t nc = w >> 63;
                w = (w << 1) | carry;
                carry = nc;
            }
            if (bit(poly_, kDegree)) {
                const Poly& q = phi().shifted[0];
                for (size_t w = 0; w < poly_.size(); ++w) poly_[w] ^= q[w];
            }
        }
    }
}

MtJump MtJump::doubled() const
{
    MtJump j;
    j.steps_ = 2 * steps_;
    Poly sq = square(poly_);
    reduce(sq);
    j.poly_ = sq;
    return j;
}

void MtJump::apply(Mt19937& g) const
{
    // Horner: sum_i a_i T^i g, from the highest coefficient down
    int deg = kDegree - 1;
    while (deg >= 0 && !bit(poly_, (size_t)deg)) --deg;
    Mt19937 r = g;
    r.clear();
    for (int i = deg; i >= 0; --i) {
        r.step();
        if (bit(poly_, (size_t)i)) r.add(g);
    }
    g = r;
}

}  // namespace MGBrain
