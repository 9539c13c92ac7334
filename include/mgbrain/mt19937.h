// MGBrain C++ API addition: the 32-bit Mersenne Twister NetGen draws from
// (the reference seeds a std::mt19937 in src/model/netgen.cpp:47), with its
// state open and a jump-ahead, so that one stretch of its output can be cut
// into pieces that threads generate at once and the result is the stream's.
//
// Mt19937 is MT19937 as published by Matsumoto and Nishimura (1998) and as
// the C++ standard defines std::mt19937: the same seed gives the same
// outputs.  It advances one word per output (the 624-word block twist
// computed word by word), so one output is one step of the linear map T on
// the state.
//
// Jump-ahead (Haramoto, Matsumoto, Nishimura, Panneton and L'Ecuyer, 2008,
// "Efficient jump ahead for F2-linear random number generators"): the
// characteristic polynomial phi of T, of degree 19937, is found once with the
// Berlekamp-Massey algorithm from 2 x 19937 output bits; advancing J outputs
// is T^J = sum a_i T^i where x^J mod phi = sum a_i x^i, evaluated on the state
// by Horner's rule (19937 steps of T).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace MGBrain {

class Mt19937 {
public:
    static constexpr int N = 624;
    explicit Mt19937(uint32_t seed = 5489u) { seed_with(seed); }
    void seed_with(uint32_t seed);
    uint32_t operator()()
    {
        step();
        return temper(x_[i_ == 0 ? N - 1 : i_ - 1]);
    }
    // the next n outputs (the same as n calls), whole blocks of 624 at once
    void generate(uint32_t* out, size_t n);
    void discard(uint64_t n);
    // One step of T: the word at the ring position is replaced by the next.
    void step()
    {
        const int i1 = i_ + 1 == N ? 0 : i_ + 1;
        const int im = i_ + 397 >= N ? i_ + 397 - N : i_ + 397;
        const uint32_t y = (x_[i_] & 0x80000000u) | (x_[i1] & 0x7fffffffu);
        x_[i_] = x_[im] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        i_ = i1;
    }
    // this ^= o, word by word in logical order (linear combination of states)
    void add(const Mt19937& o);
    void clear();
    // The state in logical order: out[k] = the word the (k+1)-th next step
    // replaces, so that the next 624 outputs are those of one block twist of
    // out[0..623] (624 words).
    void state_words(uint32_t* out) const;
    // The state from words in that order (ring position 0).
    void set_state_words(const uint32_t* in);

private:
    static uint32_t temper(uint32_t y)
    {
        y ^= y >> 11;
        y ^= (y << 7) & 0x9d2c5680u;
        y ^= (y << 15) & 0xefc60000u;
        return y ^ (y >> 18);
    }
    void twist_block();  // 624 steps from ring position 0, in three loops
    uint32_t x_[N];
    int i_ = 0;  // ring position of the oldest word (the next to be replaced)
};

// x^J mod phi as a bit vector (bit i: coefficient of x^i), 19937 bits.
class MtJump {
public:
    explicit MtJump(uint64_t steps);
    uint64_t steps() const { return steps_; }
    // g advanced by steps() outputs
    void apply(Mt19937& g) const;
    // the jump by 2 * steps() outputs (x^(2J) = (x^J)^2 mod phi)
    MtJump doubled() const;

private:
    MtJump() = default;
    uint64_t steps_ = 0;
    std::vector<uint64_t> poly_;
};

}  // namespace MGBrain
