// sdrg_gen.cu - spreading-code chip generators (host side, set-up time).
//
// Reference: src/sdr_code.c:2173-2182 (sdr_gen_code) and :2274-2283
// (sdr_sec_code) for the signals of the acquisition and tracking paths:
//   L1CA        GPS/QZSS/SBAS C/A, G1 x delayed G2 (src/sdr_code.c:794-824)
//   L5I, L5Q    GPS L5 XA x advanced XB, NH10 / NH20 overlays (:1007-1061,
//               :1100-1126)
//   L6D, L6E    QZSS L6 10-stage x 20-stage registers, time-multiplexed with
//               zeros (:1167-1212)
//   E1B         Galileo E1-B memory codes with the BOC(1,1) sub-carrier
//               (:1387-1400)
//   B1I         BeiDou G1 x phase-selected G2, NH20 overlay for D1 satellites
//               (:1613-1662)
// Chips are +1 / -1 (a 0 bit is +1), with the sub-carrier applied and zeros in
// the off slots of time-multiplexed codes, as the reference returns them.
//
// Every shift register here is described as its interface documents print
// it: a length n, the exponents of its characteristic polynomial and an
// initial state. Stage s (1..n) is bit n - s of the state word; each step
// outputs stage n, shifts every stage one place towards stage n, and loads
// stage 1 with the modulo-2 sum of the stages named by the polynomial's
// exponents. Phase-selected outputs (B1I G2) sum the named stages instead.
// Codes are generated once per (signal, PRN) and cached under a mutex.
#include <cstring>
#include <mutex>
#include <vector>

#include "sdrg_internal.h"

namespace sdrg {
namespace {

#include "sdrg_code_tables.inc"
#include "sdrg_gal_e1b.inc"

struct ShiftReg {
    int n;
    uint32_t state;
    uint32_t fb;     // stages of the feedback sum, as state bits
    ShiftReg(int n_, std::initializer_list<int> exps, uint32_t init) : n(n_), state(init), fb(0)
    {
        for (int e : exps) fb |= 1u << (n - e);
    }
    static int parity(uint32_t x) { return __builtin_parity(x); }
    int step()   // returns the output bit (stage n) before the shift
    {
        const int out = (int)(state & 1u);
        state = ((uint32_t)parity(state & fb) << (n - 1)) | (state >> 1);
        return out;
    }
};

inline int8_t chip_of(int bit) { return bit ? -1 : 1; }

std::vector<int8_t> run_reg(ShiftReg r, int len)
{
    std::vector<int8_t> c(len);
    for (int i = 0; i < len; ++i) c[i] = chip_of(r.step());
    return c;
}

// register word with stage s holding bit s-1 of `printed` (stage 1 in the
// least significant bit, as the QZSS initial states are printed)
uint32_t stages_from_printed(uint32_t printed, int n)
{
    uint32_t w = 0;
    for (int s = 1; s <= n; ++s)
        if ((printed >> (s - 1)) & 1u) w |= 1u << (n - s);
    return w;
}

// --- GPS L1 C/A (IS-GPS-200: G1 = 1 + x^3 + x^10, G2 = 1 + x^2 + x^3 + x^6 +
// x^8 + x^9 + x^10, both all ones at the start of the period) --------------
std::vector<int8_t> gen_l1ca(int prn)
{
    static const std::vector<int8_t> g1 = run_reg(ShiftReg(10, {3, 10}, 0x3FF), 1023);
    static const std::vector<int8_t> g2 = run_reg(ShiftReg(10, {2, 3, 6, 8, 9, 10}, 0x3FF), 1023);
    const int d = kL1caG2Delay[prn - 1];
    std::vector<int8_t> c(1023);
    for (int i = 0; i < 1023; ++i) c[i] = g1[i] * g2[(i + 1023 - d) % 1023];
    return c;
}

// --- GPS L5 (IS-GPS-705: XA = 1 + x^9 + x^10 + x^12 + x^13 restarted after
// 8190 chips, XB = 1 + x + x^3 + x^4 + x^6 + x^7 + x^8 + x^12 + x^13 run from
// its advanced state) -------------------------------------------------------
std::vector<int8_t> gen_l5(int prn, bool q)
{
    static const std::vector<int8_t> xa = [] {
        std::vector<int8_t> a = run_reg(ShiftReg(13, {9, 10, 12, 13}, 0x1FFF), 8190), c(10230);
        for (int i = 0; i < 10230; ++i) c[i] = a[i % 8190];
        return c;
    }();
    static const std::vector<int8_t> xb =
        run_reg(ShiftReg(13, {1, 3, 4, 6, 7, 8, 12, 13}, 0x1FFF), 10230);
    const int adv = q ? kL5qXbAdvance[prn - 1] : kL5iXbAdvance[prn - 1];
    std::vector<int8_t> c(10230);
    for (int i = 0; i < 10230; ++i) c[i] = xa[i] * xb[(i + adv) % 10230];
    return c;
}

// --- QZSS L6 (IS-QZSS-L6: 10-stage 1 + x^3 + x^4 + x^5 + x^6 + x^9 + x^10 from
// all ones, times the 20-stage 1 + x^14 + x^16 + x^19 + x^20 register from the
// PRN's initial state; L6D in the even chip slots, L6E in the odd ones) -----
std::vector<int8_t> gen_l6(uint32_t printed_init, int slot)
{
    static const std::vector<int8_t> a = run_reg(ShiftReg(10, {3, 4, 5, 6, 9, 10}, 0x3FF), 10230);
    const std::vector<int8_t> b =
        run_reg(ShiftReg(20, {14, 16, 19, 20}, stages_from_printed(printed_init, 20)), 10230);
    std::vector<int8_t> c(2 * 10230, 0);
    for (int i = 0; i < 10230; ++i) c[2 * i + slot] = a[i] * b[i];
    return c;
}

// --- Galileo E1-B (OS SIS ICD annex C memory code, BOC(1,1) sub-carrier as
// +1, -1 half chips; the reference uses BOC(1,1) in place of CBOC) ----------
std::vector<int8_t> gen_e1b(int prn)
{
    const char *hex = kGalE1BHex[prn - 1];
    std::vector<int8_t> c(2 * 4092);
    for (int i = 0; i < 4092; ++i) {
        const char h = hex[i / 4];
        const int v = (h >= '0' && h <= '9') ? h - '0' : h - 'A' + 10;
        const int8_t chip = chip_of((v >> (3 - i % 4)) & 1);
        c[2 * i] = chip;
        c[2 * i + 1] = (int8_t)-chip;
    }
    return c;
}

// --- BeiDou B1I (BDS-SIS-ICD-B1I: G1 = 1 + x + x^7 + x^8 + x^9 + x^10 + x^11,
// G2 = 1 + x + x^2 + x^3 + x^4 + x^5 + x^8 + x^9 + x^11, both from 01010101010;
// G2's output is the sum of the PRN's selected stages) ----------------------
std::vector<int8_t> gen_b1i(int prn)
{
    static const std::vector<int8_t> g1 =
        run_reg(ShiftReg(11, {1, 7, 8, 9, 10, 11}, 0x2AA), 2046);
    ShiftReg g2(11, {1, 2, 3, 4, 5, 8, 9, 11}, 0x2AA);
    uint32_t sel = 0;
    for (int k = 0; k < 3 && kB1iPhaseSel[prn - 1][k]; ++k) sel |= 1u << (11 - kB1iPhaseSel[prn - 1][k]);
    std::vector<int8_t> c(2046);
    for (int i = 0; i < 2046; ++i) {
        const int bit = ShiftReg::parity(g2.state & sel);
        g2.step();
        c[i] = g1[i] * chip_of(bit);
    }
    return c;
}

// Neuman-Hoffman overlays (IS-GPS-705 3.3.2.1: NH10 = 0000110101, NH20 =
// 00000100110101001110), the SBAS L5 Manchester overlay (01)
std::vector<int8_t> bits_to_chips(const char *bits)
{
    std::vector<int8_t> c;
    for (const char *p = bits; *p; ++p) c.push_back(chip_of(*p == '1'));
    return c;
}

enum Sig { kNone, kL1CA, kL5I, kL5Q, kL6D, kL6E, kE1B, kB1I };

Sig sig_of(const char *sig)
{
    if (!sig) return kNone;
    char s[16];
    int i = 0;
    for (; i < 15 && sig[i]; ++i) s[i] = (char)(sig[i] >= 'a' && sig[i] <= 'z' ? sig[i] - 32 : sig[i]);
    s[i] = 0;
    static const struct { const char *name; Sig v; } names[] = {
        {"L1CA", kL1CA}, {"L5I", kL5I}, {"L5Q", kL5Q}, {"L6D", kL6D},
        {"L6E", kL6E}, {"E1B", kE1B}, {"B1I", kB1I}};
    for (const auto &n : names)
        if (!strcmp(s, n.name)) return n.v;
    return kNone;
}

bool prn_ok(Sig s, int prn)
{
    switch (s) {
    case kL1CA: case kL5I: case kL5Q: return prn >= 1 && prn <= 210;
    case kL6D: return prn >= 193 && prn <= 202;
    case kL6E: return prn >= 203 && prn <= 212;
    case kE1B: return prn >= 1 && prn <= 50;
    case kB1I: return prn >= 1 && prn <= 63;
    default: return false;
    }
}

std::mutex g_gen_mtx;
std::vector<int8_t> g_cache[8][213];   // [signal][prn]

const std::vector<int8_t> &primary(Sig s, int prn)
{
    std::vector<int8_t> &c = g_cache[s][prn];
    if (c.empty()) {
        switch (s) {
        case kL1CA: c = gen_l1ca(prn); break;
        case kL5I: c = gen_l5(prn, false); break;
        case kL5Q: c = gen_l5(prn, true); break;
        case kL6D: c = gen_l6(kL6dInit[prn - 193], 0); break;
        case kL6E: c = gen_l6(kL6eInit[prn - 203], 1); break;
        case kE1B: c = gen_e1b(prn); break;
        case kB1I: c = gen_b1i(prn); break;
        default: break;
        }
    }
    return c;
}

std::vector<int8_t> secondary(Sig s, int prn)
{
    static const std::vector<int8_t> nh10 = bits_to_chips("0000110101");
    static const std::vector<int8_t> nh20 = bits_to_chips("00000100110101001110");
    static const std::vector<int8_t> manchester = bits_to_chips("01");
    const bool sbas = prn >= 120 && prn <= 158;
    switch (s) {
    case kL5I: return sbas ? manchester : nh10;
    case kL5Q: return sbas ? manchester : nh20;
    case kB1I: return (prn >= 6 && prn <= 58) ? nh20 : std::vector<int8_t>{1};   // D1 / D2 (GEO)
    default: return {1};
    }
}

int copy_out(const std::vector<int8_t> &c, int8_t *out, int cap, const char *what)
{
    if (out) {
        if (cap < (int)c.size())
            return set_error(SDRG_ERR_ARG, "%s: %d chips do not fit %d", what, (int)c.size(), cap);
        memcpy(out, c.data(), c.size());
    }
    return (int)c.size();
}

} // namespace
} // namespace sdrg

using namespace sdrg;

extern "C" {

int sdrg_gen_code(const char *sig, int prn, int8_t *chips, int cap)
{
    const Sig s = sig_of(sig);
    if (s == kNone || !prn_ok(s, prn))
        return set_error(SDRG_ERR_ARG, "sdrg_gen_code: no code for %s PRN %d", sig ? sig : "(null)", prn);
    std::lock_guard<std::mutex> lk(g_gen_mtx);
    return copy_out(primary(s, prn), chips, cap, "sdrg_gen_code");
}

int sdrg_sec_code(const char *sig, int prn, int8_t *chips, int cap)
{
    const Sig s = sig_of(sig);
    if (s == kNone || !prn_ok(s, prn))
        return set_error(SDRG_ERR_ARG, "sdrg_sec_code: no code for %s PRN %d", sig ? sig : "(null)", prn);
    return copy_out(secondary(s, prn), chips, cap, "sdrg_sec_code");
}

} // extern "C"
