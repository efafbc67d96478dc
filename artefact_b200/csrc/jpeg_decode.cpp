// Host-side baseline JPEG coefficient decoder.
//
// Stands in for the zune-jpeg fork that artefact-lib uses on the host
// (backend/zune-jpeg/src/decoder.rs:187-206, mcu.rs:80-290, bitstream.rs:326-390,
// headers.rs:115-178) and produces the same solver-input contract as
// backend/artefact-lib/jpeg/zune.rs:22-46:
//   * per component: rounded_px_w/h = image size rounded up to 8 * max sampling
//     factor, divided by the component's sampling factor (misc.rs:209-249);
//   * samp_h/samp_v = max sampling / component sampling (1 or 2);
//   * quantised coefficients as int16 in natural (row-major, v*8+u) order within
//     each 8x8 block, blocks in raster order over the component plane;
//   * quantisation tables in natural order.
// Sequential (SOF0/SOF1) and progressive (SOF2) Huffman coding, 8-bit samples,
// restart markers, interleaved or single-component scans. Progressive scans
// follow ITU-T T.81 Annex G (zune-jpeg's mcu_prog.rs decodes the same
// streams): DC first/refinement scans, AC spectral-selection first scans with
// end-of-band runs, and AC successive-approximation refinement; the
// coefficients accumulate over the scans into the same output contract.
// Arithmetic-coded, lossless and hierarchical streams are rejected.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "art_internal.h"

namespace art {

namespace {

const uint8_t kZigzagToNatural[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
    41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
    30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct DecodeError {
    std::string msg;
};

[[noreturn]] void fail(const std::string &m) { throw DecodeError{m}; }

struct Huffman {
    bool present = false;
    // Canonical code description (ITU T.81 Annex C / F.2.2.3).
    int32_t maxcode[18];
    int32_t valptr[17];
    int32_t mincode[17];
    uint8_t vals[256];
    // 9-bit lookahead: (length << 8) | value, 0 when the code is longer.
    uint16_t fast[512];
    // AC tables: 11-bit lookahead decoding a code and its magnitude bits at
    // once (see ac_entry); empty for DC tables.
    std::vector<uint32_t> fast_ac;
};

// Combined AC lookahead entries: bits 0-4 the bits consumed, 5-8 the run,
// 9-10 the kind (1: a coefficient whose value is in bits 16-31, 2: a size-0
// symbol with run r < 15 -- end of block, or in a progressive scan the start
// of an end-of-band run; 0: no shortcut -- a longer code, ZRL, or magnitude
// bits beyond the window), 16-31 the sign-extended coefficient.
constexpr int AC_LOOK = 11;
constexpr uint32_t AC_COEF = 1u << 9, AC_EOB = 2u << 9;

static inline int extend(int v, int t) { return v < (1 << (t - 1)) ? v - (1 << t) + 1 : v; }

void build_huffman(Huffman &h, const uint8_t counts[16], const uint8_t *symbols, int nsym, bool ac)
{
    h.present = false;
    memset(h.maxcode, 0, sizeof(h.maxcode));
    memset(h.valptr, 0, sizeof(h.valptr));
    memset(h.mincode, 0, sizeof(h.mincode));
    memset(h.vals, 0, sizeof(h.vals));
    memset(h.fast, 0, sizeof(h.fast));
    h.fast_ac.clear();
    memcpy(h.vals, symbols, nsym);
    int code = 0, k = 0;
    for (int len = 1; len <= 16; len++) {
        h.valptr[len] = k;
        h.mincode[len] = code;
        code += counts[len - 1];
        k += counts[len - 1];
        h.maxcode[len] = counts[len - 1] ? code - 1 : -1;
        if (code > (1 << len)) fail("Invalid Huffman table: code space overflow");
        code <<= 1;
    }
    h.maxcode[17] = 0x7fffffff;
    // Fill the lookahead table.
    k = 0;
    code = 0;
    for (int len = 1; len <= 9; len++) {
        for (int i = 0; i < counts[len - 1]; i++, k++) {
            int c = h.mincode[len] + i;
            int shift = 9 - len;
            for (int f = 0; f < (1 << shift); f++) h.fast[(c << shift) | f] = (uint16_t)((len << 8) | symbols[k]);
        }
    }
    if (ac) {
        h.fast_ac.assign(1u << AC_LOOK, 0u);
        k = 0;
        for (int len = 1; len <= AC_LOOK; len++) {
            for (int i = 0; i < counts[len - 1]; i++, k++) {
                const int c = h.mincode[len] + i, rs = symbols[k], r = rs >> 4, sz = rs & 15;
                const int shift = AC_LOOK - len;
                for (int f = 0; f < (1 << shift); f++) {
                    uint32_t e = 0;
                    if (sz == 0) {
                        if (r != 15) e = (uint32_t)len | ((uint32_t)r << 5) | AC_EOB;  // ZRL: general path
                    } else if (len + sz <= AC_LOOK) {
                        const int mag = f >> (shift - sz);  // the sz bits after the code
                        const int v = extend(mag, sz);
                        e = (uint32_t)(len + sz) | ((uint32_t)r << 5) | AC_COEF | ((uint32_t)(uint16_t)(int16_t)v << 16);
                    }
                    h.fast_ac[(c << shift) | f] = e;
                }
            }
        }
    }
    h.present = true;
}

struct Component {
    int id = 0;
    int h = 1, v = 1, tq = 0;
    int td = 0, ta = 0;
    int dc_pred = 0;
    uint32_t rounded_w = 0, rounded_h = 0, block_w = 0, block_h = 0;
    CoefVec coefs;
    bool defined = false;  // every element of coefs has been written (else they are uninitialised)
};

class Decoder {
  public:
    Decoder(const uint8_t *data, size_t len) : d_(data), n_(len) {}

    void run(JpegImage &out);

  private:
    const uint8_t *d_;
    size_t n_;
    size_t pos_ = 0;
    uint16_t qt_[4][64];
    bool qt_present_[4] = {false, false, false, false};
    Huffman dc_[4], ac_[4];
    std::vector<Component> comps_;
    bool have_sof_ = false;
    bool progressive_ = false;
    int eobrun_ = 0;  // progressive AC scans: blocks left in the current end-of-band run
    int width_ = 0, height_ = 0;
    int hmax_ = 1, vmax_ = 1;
    int restart_interval_ = 0;
    // Bit reader state: the next bitcnt_ bits of the entropy-coded data,
    // MSB-aligned in a 64-bit word.
    uint64_t bitbuf_ = 0;
    int bitcnt_ = 0;
    bool hit_marker_ = false;

    uint8_t u8()
    {
        if (pos_ >= n_) fail("No more bytes: unexpected end of JPEG stream");
        return d_[pos_++];
    }
    uint16_t u16()
    {
        uint16_t a = u8();
        return (uint16_t)((a << 8) | u8());
    }
    void parse_dqt();
    void parse_dht();
    void parse_sof(int marker);
    void parse_sos();
    void decode_scan(const std::vector<int> &scomp);
    void decode_scan_progressive(const std::vector<int> &scomp, int ss, int se, int ah, int al);
    void prog_dc_first(Component &c, int16_t *blk, int al);
    void prog_dc_refine(int16_t *blk, int al);
    void prog_ac_first(Component &c, int16_t *blk, int ss, int se, int al);
    void prog_ac_refine(Component &c, int16_t *blk, int ss, int se, int al);
    void fill_bits();
    int get_bits(int n);
    int decode_huff(const Huffman &h);
    int decode_huff_nofill(const Huffman &h);
    int take_bits(int n)  // n <= bitcnt_, 1 <= n <= 16
    {
        const int v = (int)(bitbuf_ >> (64 - n));
        bitbuf_ <<= n;
        bitcnt_ -= n;
        return v;
    }
    void decode_block(Component &c, int16_t *blk);
    void reset_bits()
    {
        bitbuf_ = 0;
        bitcnt_ = 0;
        hit_marker_ = false;
    }
    void handle_restart();
};

void Decoder::parse_dqt()
{
    int len = u16();
    if (len < 2) fail("Invalid DQT length. Length should be greater than 2");
    len -= 2;
    while (len > 0) {
        int info = u8();
        int prec = info >> 4, id = info & 15;
        int need = 64 * (prec + 1) + 1;
        if (need > len) fail("Invalid QT table: too few bytes left");
        if (prec > 1) fail("Expected QT precision value of either 0 or 1");
        if (id >= 4) fail("Too large table position for QT");
        for (int i = 0; i < 64; i++) qt_[id][kZigzagToNatural[i]] = prec ? u16() : u8();
        qt_present_[id] = true;
        len -= need;
    }
}

void Decoder::parse_dht()
{
    int len = u16();
    if (len < 2) fail("Invalid Huffman length in image");
    len -= 2;
    while (len > 0) {
        if (len < 17) fail("Invalid Huffman length in image");
        int info = u8();
        int tc = info >> 4, th = info & 15;
        if (tc > 1 || th > 3) fail("Invalid Huffman table class or index");
        uint8_t counts[16];
        int total = 0;
        for (int i = 0; i < 16; i++) {
            counts[i] = u8();
            total += counts[i];
        }
        if (total > 256 || 17 + total > len) fail("Invalid Huffman length in image");
        uint8_t syms[256];
        for (int i = 0; i < total; i++) syms[i] = u8();
        build_huffman(tc ? ac_[th] : dc_[th], counts, syms, total, tc != 0);
        len -= 17 + total;
    }
}

void Decoder::parse_sof(int marker)
{
    if (marker == 0xC6 || marker == 0xCA || marker == 0xCE)
        fail("Differential or arithmetic progressive JPEG is not supported by this decoder");
    if (marker != 0xC0 && marker != 0xC1 && marker != 0xC2)
        fail("Unsupported JPEG coding process (lossless or arithmetic)");
    progressive_ = marker == 0xC2;
    if (have_sof_) fail("Duplicate start of frame");
    int len = u16();
    int prec = u8();
    height_ = u16();
    width_ = u16();
    int nc = u8();
    int expected = 8 + 3 * nc;
    if (len != expected)
        fail("Length of start of frame differs from expected " + std::to_string(expected) + ",value is " +
             std::to_string(len));
    if (prec != 8) fail("Only 8-bit sample precision is supported");
    if (width_ == 0 || height_ == 0) fail("Zero image dimension");
    if (nc != 1 && nc != 3 && nc != 4) fail("Unsupported number of components");
    comps_.resize(nc);
    for (int i = 0; i < nc; i++) {
        Component &c = comps_[i];
        c.id = u8();
        int hv = u8();
        c.h = hv >> 4;
        c.v = hv & 15;
        c.tq = u8();
        if (c.h < 1 || c.h > 2 || c.v < 1 || c.v > 2) fail("Unknown sample factor, expected either 1 or 2");
        if (c.tq > 3) fail("Invalid quantization table index");
    }
    if (nc == 1) comps_[0].h = comps_[0].v = 1;  // single-component scans are never interleaved
    hmax_ = vmax_ = 1;
    for (auto &c : comps_) {
        if (c.h > hmax_) hmax_ = c.h;
        if (c.v > vmax_) vmax_ = c.v;
    }
    // misc.rs:209-249: round to 8 * max sampling, then divide by the component's factor.
    uint32_t mw = 8 * hmax_ - 1, mh = 8 * vmax_ - 1;
    uint32_t rw = ((uint32_t)width_ + mw) & ~mw;
    uint32_t rh = ((uint32_t)height_ + mh) & ~mh;
    for (auto &c : comps_) {
        int sf_h = hmax_ / c.h, sf_v = vmax_ / c.v;
        c.rounded_w = rw / sf_h;
        c.rounded_h = rh / sf_v;
        c.block_w = c.rounded_w / 8;
        c.block_h = c.rounded_h / 8;
        // Progressive scans refine what earlier scans left, so they start from
        // zeros. A sequential scan writes each block it codes in full (zeros
        // included); blocks no scan codes are zeroed when that is known.
        if (progressive_) {
            c.coefs.assign((size_t)c.rounded_w * c.rounded_h, 0);
            c.defined = true;
        } else {
            c.coefs.resize((size_t)c.rounded_w * c.rounded_h);
            c.defined = false;
        }
    }
    have_sof_ = true;
}

// Tops the buffer up to at least 57 bits. Byte stuffing (FF 00) is undone;
// at a marker (FF followed by anything else) the reader stops in front of it
// and feeds zero bytes from then on (T.81 F.2.2.5). Eight bytes without an FF
// are appended in one step.
void Decoder::fill_bits()
{
    if (!hit_marker_ && bitcnt_ <= 56 && pos_ + 8 <= n_) {
        uint64_t w;
        memcpy(&w, d_ + pos_, 8);
        const uint64_t x = ~w;  // a byte of w is FF exactly when this byte of x is 0
        if (!((x - 0x0101010101010101ULL) & ~x & 0x8080808080808080ULL)) {
            const int nb = (64 - bitcnt_) >> 3;  // whole bytes that fit: 1..8
            const uint64_t be = __builtin_bswap64(w);  // first byte of the stream in the top byte
            bitbuf_ |= (be >> (64 - 8 * nb)) << (64 - 8 * nb - bitcnt_);
            pos_ += (size_t)nb;
            bitcnt_ += 8 * nb;
            return;
        }
    }
    while (bitcnt_ <= 56) {
        uint64_t byte = 0;
        if (!hit_marker_ && pos_ < n_) {
            byte = d_[pos_];
            if (byte == 0xFF) {
                uint8_t next = pos_ + 1 < n_ ? d_[pos_ + 1] : 0xD9;
                if (next == 0x00) {
                    pos_ += 2;
                } else {
                    hit_marker_ = true;  // leave the marker in place, feed zeros
                    byte = 0;
                }
            } else {
                pos_++;
            }
        }
        bitbuf_ |= byte << (56 - bitcnt_);
        bitcnt_ += 8;
    }
}

int Decoder::get_bits(int n)
{
    if (n == 0) return 0;
    if (bitcnt_ < n) fill_bits();
    return take_bits(n);
}

// Huffman symbol from a buffer holding at least 16 bits.
int Decoder::decode_huff_nofill(const Huffman &h)
{
    const uint16_t f = h.fast[bitbuf_ >> 55];
    if (f) {
        const int l = f >> 8;
        bitbuf_ <<= l;
        bitcnt_ -= l;
        return f & 0xFF;
    }
    int code = 0;
    for (int len = 1; len <= 16; len++) {
        code = (code << 1) | (int)(bitbuf_ >> 63);
        bitbuf_ <<= 1;
        bitcnt_--;
        if (h.maxcode[len] >= 0 && code <= h.maxcode[len] && code >= h.mincode[len])
            return h.vals[h.valptr[len] + code - h.mincode[len]];
    }
    fail("Bad Huffman code: corrupt JPEG entropy data");
}

int Decoder::decode_huff(const Huffman &h)
{
    if (bitcnt_ < 16) fill_bits();
    return decode_huff_nofill(h);
}

// One block of a sequential scan into blk (zeroed here). The buffer is
// topped up to 32+ bits before each Huffman code, which leaves 16+ bits for
// the code's magnitude bits (at most 15).
void Decoder::decode_block(Component &c, int16_t *blk)
{
    const Huffman &dc = dc_[c.td], &ac = ac_[c.ta];
    memset(blk, 0, 64 * sizeof(int16_t));
    if (bitcnt_ < 32) fill_bits();
    int t = decode_huff_nofill(dc);
    if (t > 11) fail("Bad DC magnitude category");
    int diff = t ? extend(take_bits(t), t) : 0;
    c.dc_pred += diff;
    blk[0] = (int16_t)c.dc_pred;
    const uint32_t *fast_ac = ac.fast_ac.data();
    for (int k = 1; k < 64;) {
        if (bitcnt_ < 32) fill_bits();
        const uint32_t e = fast_ac[bitbuf_ >> (64 - AC_LOOK)];
        if (e & AC_COEF) {  // code and magnitude bits in one step
            k += (int)((e >> 5) & 15);
            if (k > 63) fail("Coefficient index out of range: corrupt JPEG");
            blk[kZigzagToNatural[k]] = (int16_t)(e >> 16);
            const int l = (int)(e & 31);
            bitbuf_ <<= l;
            bitcnt_ -= l;
            k++;
            continue;
        }
        if (e & AC_EOB) {
            const int l = (int)(e & 31);
            bitbuf_ <<= l;
            bitcnt_ -= l;
            break;
        }
        int rs = decode_huff_nofill(ac);
        int r = rs >> 4, s = rs & 15;
        if (s == 0) {
            if (r != 15) break;  // EOB
            k += 16;
            continue;
        }
        k += r;
        if (k > 63) fail("Coefficient index out of range: corrupt JPEG");
        blk[kZigzagToNatural[k]] = (int16_t)extend(take_bits(s), s);
        k++;
    }
}

void Decoder::handle_restart()
{
    // Discard buffered bits, then expect RSTn.
    reset_bits();
    while (pos_ + 1 < n_ && !(d_[pos_] == 0xFF && d_[pos_ + 1] >= 0xD0 && d_[pos_ + 1] <= 0xD7)) {
        if (d_[pos_] == 0xFF && d_[pos_ + 1] != 0x00 && d_[pos_ + 1] != 0xFF) break;
        pos_++;
    }
    if (pos_ + 1 < n_ && d_[pos_] == 0xFF && d_[pos_ + 1] >= 0xD0 && d_[pos_ + 1] <= 0xD7) pos_ += 2;
    for (auto &c : comps_) c.dc_pred = 0;
}

void Decoder::decode_scan(const std::vector<int> &scomp)
{
    reset_bits();
    for (auto &c : comps_) c.dc_pred = 0;
    int todo = restart_interval_;
    if (scomp.size() == 1) {
        // Non-interleaved: blocks covering ceil(component samples / 8).
        Component &c = comps_[scomp[0]];
        int cw = (width_ * c.h + hmax_ - 1) / hmax_, chh = (height_ * c.v + vmax_ - 1) / vmax_;
        int bw = (cw + 7) / 8, bh = (chh + 7) / 8;
        if (!c.defined) {
            // Blocks of the rounded plane that this scan does not code stay zero.
            for (uint32_t by = 0; by < c.block_h; by++)
                for (uint32_t bx = (by < (uint32_t)bh ? (uint32_t)bw : 0); bx < c.block_w; bx++)
                    memset(&c.coefs[((size_t)by * c.block_w + bx) * 64], 0, 64 * sizeof(int16_t));
            c.defined = true;
        }
        for (int by = 0; by < bh; by++)
            for (int bx = 0; bx < bw; bx++) {
                if (restart_interval_ && todo == 0) {
                    handle_restart();
                    todo = restart_interval_;
                }
                int16_t pad[64];  // blocks past the component's rounded size are decoded and dropped
                const bool in = (uint32_t)bx < c.block_w && (uint32_t)by < c.block_h;
                decode_block(c, in ? &c.coefs[((size_t)by * c.block_w + bx) * 64] : pad);
                if (restart_interval_) todo--;
            }
        return;
    }
    int mcu_w = (width_ + 8 * hmax_ - 1) / (8 * hmax_), mcu_h = (height_ + 8 * vmax_ - 1) / (8 * vmax_);
    // The MCUs of an interleaved scan cover every block of its components'
    // rounded planes (block_w = mcu_w * h, block_h = mcu_h * v).
    for (int ci : scomp) comps_[ci].defined = true;
    for (int my = 0; my < mcu_h; my++)
        for (int mx = 0; mx < mcu_w; mx++) {
            if (restart_interval_ && todo == 0) {
                handle_restart();
                todo = restart_interval_;
            }
            for (int ci : scomp) {
                Component &c = comps_[ci];
                for (int v = 0; v < c.v; v++)
                    for (int u = 0; u < c.h; u++) {
                        int16_t pad[64];  // blocks past the component's rounded size are decoded and dropped
                        const uint32_t bx = (uint32_t)(mx * c.h + u), by = (uint32_t)(my * c.v + v);
                        const bool in = bx < c.block_w && by < c.block_h;
                        decode_block(c, in ? &c.coefs[((size_t)by * c.block_w + bx) * 64] : pad);
                    }
            }
            if (restart_interval_) todo--;
        }
}

// Progressive DC first scan: the DC difference as in a sequential scan, the
// coefficient stored shifted left by the scan's point transform Al (G.1.2.1).
void Decoder::prog_dc_first(Component &c, int16_t *blk, int al)
{
    const Huffman &dc = dc_[c.td];
    if (!dc.present) fail("No DC table for component");
    int t = decode_huff(dc);
    if (t > 11) fail("Bad DC magnitude category");
    int diff = t ? extend(get_bits(t), t) : 0;
    c.dc_pred += diff;
    blk[0] = (int16_t)(c.dc_pred * (1 << al));
}

// Progressive DC refinement: one more bit of the DC coefficient (G.1.2.1).
void Decoder::prog_dc_refine(int16_t *blk, int al)
{
    if (get_bits(1)) blk[0] = (int16_t)(blk[0] | (1 << al));
}

// Progressive AC first scan over zigzag positions ss..se (G.1.2.2): run/size
// symbols as in a sequential scan, values shifted by Al; a symbol with size 0
// and run r < 15 starts an end-of-band run of 2^r + (r extra bits) - 1 more
// blocks whose band is all zero.
void Decoder::prog_ac_first(Component &c, int16_t *blk, int ss, int se, int al)
{
    if (eobrun_ > 0) {
        eobrun_--;
        return;
    }
    const Huffman &ac = ac_[c.ta];
    if (!ac.present) fail("No AC table for component");
    const uint32_t *fast_ac = ac.fast_ac.data();
    for (int k = ss; k <= se;) {
        if (bitcnt_ < 32) fill_bits();
        const uint32_t e = fast_ac[bitbuf_ >> (64 - AC_LOOK)];
        if (e & AC_COEF) {  // code and magnitude bits in one step
            k += (int)((e >> 5) & 15);
            if (k > se) fail("Coefficient index out of range: corrupt JPEG");
            blk[kZigzagToNatural[k]] = (int16_t)((int32_t)(int16_t)(e >> 16) * (1 << al));
            const int l = (int)(e & 31);
            bitbuf_ <<= l;
            bitcnt_ -= l;
            k++;
            continue;
        }
        if ((e & AC_EOB) && ((e >> 5) & 15) == 0) {  // end of band, no run
            const int l = (int)(e & 31);
            bitbuf_ <<= l;
            bitcnt_ -= l;
            break;
        }
        int rs = decode_huff_nofill(ac);
        int r = rs >> 4, sz = rs & 15;
        if (sz == 0) {
            if (r < 15) {
                eobrun_ = (1 << r) - 1;
                if (r) eobrun_ += get_bits(r);
                break;
            }
            k += 16;
            continue;
        }
        k += r;
        if (k > se) fail("Coefficient index out of range: corrupt JPEG");
        blk[kZigzagToNatural[k]] = (int16_t)(extend(get_bits(sz), sz) * (1 << al));
        k++;
    }
}

// Progressive AC refinement over zigzag positions ss..se (G.1.2.3). Each
// coefficient already non-zero gets one correction bit (adding 2^Al in its
// own sign's direction when set and that bit is not yet in it); the zero run
// of a symbol counts only coefficients still zero, and the symbol's new
// coefficient (size 1: +-2^Al by one sign bit) lands on the zero after that
// run. Inside an end-of-band run only the correction bits are read.
void Decoder::prog_ac_refine(Component &c, int16_t *blk, int ss, int se, int al)
{
    const int p1 = 1 << al, m1 = -(1 << al);
    auto correct = [&](int16_t &coef) {
        if (get_bits(1) && (coef & p1) == 0) coef = (int16_t)(coef + (coef >= 0 ? p1 : m1));
    };
    int k = ss;
    if (eobrun_ == 0) {
        const Huffman &ac = ac_[c.ta];
        if (!ac.present) fail("No AC table for component");
        for (; k <= se;) {
            int rs = decode_huff(ac);
            int r = rs >> 4, sz = rs & 15;
            int value = 0;
            if (sz) {
                if (sz != 1) fail("Bad AC refinement symbol: corrupt JPEG");
                value = get_bits(1) ? p1 : m1;
            } else if (r != 15) {
                eobrun_ = 1 << r;
                if (r) eobrun_ += get_bits(r);
                break;  // the rest of this block is in the end-of-band run
            }
            // Skip r still-zero coefficients (correcting the non-zero ones
            // passed on the way), then place `value` on the next zero.
            while (k <= se) {
                int16_t &coef = blk[kZigzagToNatural[k]];
                if (coef != 0) {
                    correct(coef);
                } else {
                    if (r == 0) {
                        if (value) coef = (int16_t)value;
                        k++;
                        break;
                    }
                    r--;
                }
                k++;
            }
        }
    }
    if (eobrun_ > 0) {
        for (; k <= se; k++) {
            int16_t &coef = blk[kZigzagToNatural[k]];
            if (coef != 0) correct(coef);
        }
        eobrun_--;
    }
}

// One progressive scan: DC scans may interleave components (MCU order as in a
// sequential scan); AC scans cover one component in its own block order.
void Decoder::decode_scan_progressive(const std::vector<int> &scomp, int ss, int se, int ah, int al)
{
    reset_bits();
    for (auto &c : comps_) c.dc_pred = 0;
    eobrun_ = 0;
    int todo = restart_interval_;
    auto restart_if_due = [&]() {
        if (restart_interval_ && todo == 0) {
            handle_restart();
            eobrun_ = 0;
            todo = restart_interval_;
        }
    };
    auto one_block = [&](Component &c, uint32_t bx, uint32_t by) {
        int16_t scratch[64];
        const bool inside = bx < c.block_w && by < c.block_h;
        if (!inside) memset(scratch, 0, sizeof(scratch));  // blocks past the rounded plane are decoded and dropped
        int16_t *blk = inside ? &c.coefs[((size_t)by * c.block_w + bx) * 64] : scratch;
        if (ss == 0) {
            if (ah == 0)
                prog_dc_first(c, blk, al);
            else
                prog_dc_refine(blk, al);
        } else if (ah == 0) {
            prog_ac_first(c, blk, ss, se, al);
        } else {
            prog_ac_refine(c, blk, ss, se, al);
        }
    };
    if (scomp.size() == 1) {
        Component &c = comps_[scomp[0]];
        int cw = (width_ * c.h + hmax_ - 1) / hmax_, chh = (height_ * c.v + vmax_ - 1) / vmax_;
        int bw = (cw + 7) / 8, bh = (chh + 7) / 8;
        for (int by = 0; by < bh; by++)
            for (int bx = 0; bx < bw; bx++) {
                restart_if_due();
                one_block(c, (uint32_t)bx, (uint32_t)by);
                if (restart_interval_) todo--;
            }
        return;
    }
    int mcu_w = (width_ + 8 * hmax_ - 1) / (8 * hmax_), mcu_h = (height_ + 8 * vmax_ - 1) / (8 * vmax_);
    // The MCUs of an interleaved scan cover every block of its components'
    // rounded planes (block_w = mcu_w * h, block_h = mcu_h * v).
    for (int ci : scomp) comps_[ci].defined = true;
    for (int my = 0; my < mcu_h; my++)
        for (int mx = 0; mx < mcu_w; mx++) {
            restart_if_due();
            for (int ci : scomp) {
                Component &c = comps_[ci];
                for (int v = 0; v < c.v; v++)
                    for (int u = 0; u < c.h; u++) one_block(c, (uint32_t)(mx * c.h + u), (uint32_t)(my * c.v + v));
            }
            if (restart_interval_) todo--;
        }
}

void Decoder::parse_sos()
{
    int len = u16();
    if (!have_sof_) {
        if (len < 6 || len > 10) fail("Bad SOS length " + std::to_string(len) + ",corrupt jpeg");
        fail("Scan found before start of frame");
    }
    int ns = u8();
    if (ns < 1 || ns > 4 || len != 6 + 2 * ns) fail("Bad SOS length " + std::to_string(len) + ",corrupt jpeg");
    std::vector<int> scomp;
    for (int i = 0; i < ns; i++) {
        int cid = u8();
        int t = u8();
        int idx = -1;
        for (size_t k = 0; k < comps_.size(); k++)
            if (comps_[k].id == cid) idx = (int)k;
        if (idx < 0) fail("Scan references an unknown component");
        comps_[idx].td = t >> 4;
        comps_[idx].ta = t & 15;
        if (comps_[idx].td > 3 || comps_[idx].ta > 3) fail("Invalid Huffman table index in scan");
        if (!progressive_) {
            if (!dc_[comps_[idx].td].present) fail("No DC table for component");
            if (!ac_[comps_[idx].ta].present) fail("No AC table for component");
        }
        scomp.push_back(idx);
    }
    int ss = u8(), se = u8(), ahal = u8();
    if (!progressive_) {
        if (ss != 0 || se != 63 || ahal != 0) fail("Invalid spectral selection for a sequential scan");
        decode_scan(scomp);
        return;
    }
    const int ah = ahal >> 4, al = ahal & 15;
    if (se > 63 || ss > se || (ss == 0 && se != 0) || (ss > 0 && ns != 1) || al > 13 || ah > 13)
        fail("Invalid progressive scan parameters");
    decode_scan_progressive(scomp, ss, se, ah, al);
}

void Decoder::run(JpegImage &out)
{
    if (n_ < 2 || d_[0] != 0xFF || d_[1] != 0xD8) fail("Not a JPEG file: missing SOI marker");
    pos_ = 2;
    bool done = false;
    while (!done) {
        uint8_t b = u8();
        if (b != 0xFF) fail("Expected a marker, found byte " + std::to_string(b));
        uint8_t m = u8();
        while (m == 0xFF) m = u8();
        switch (m) {
        case 0x00: fail("Bad marker 0xFF00 outside entropy-coded data");
        case 0xD8: fail("Duplicate SOI marker");
        case 0xD9: done = true; break;
        case 0xDB: parse_dqt(); break;
        case 0xC4: parse_dht(); break;
        case 0xDD: {
            int len = u16();
            if (len != 4) fail("Bad DRI length");
            restart_interval_ = u16();
            break;
        }
        case 0xDA: parse_sos(); break;
        case 0xC0: case 0xC1: case 0xC2: case 0xC3: case 0xC5: case 0xC6: case 0xC7:
        case 0xC9: case 0xCA: case 0xCB: case 0xCD: case 0xCE: case 0xCF:
            parse_sof(m);
            break;
        default:
            if (m >= 0xD0 && m <= 0xD7) break;  // stray RST
            {
                int len = u16();
                if (len < 2) fail("Bad marker segment length");
                if (pos_ + (size_t)(len - 2) > n_) fail("No more bytes: unexpected end of JPEG stream");
                pos_ += (size_t)(len - 2);
            }
        }
        if (!done && pos_ >= n_) {
            if (have_sof_) done = true;  // tolerate a missing EOI after decoded scans
            else fail("No more bytes: unexpected end of JPEG stream");
        }
    }
    if (!have_sof_) fail("No start of frame found");
    out.real_w = (uint32_t)width_;
    out.real_h = (uint32_t)height_;
    out.channels.clear();
    for (auto &c : comps_) {
        if (!qt_present_[c.tq]) fail("No quantization table for component");
        JpegChannel jc;
        jc.rounded_px_w = c.rounded_w;
        jc.rounded_px_h = c.rounded_h;
        jc.block_w = c.block_w;
        jc.block_h = c.block_h;
        jc.samp_h = (uint32_t)(hmax_ / c.h);
        jc.samp_v = (uint32_t)(vmax_ / c.v);
        for (int j = 0; j < 64; j++) jc.quant[j] = (float)qt_[c.tq][j];
        if (!c.defined) c.coefs.assign(c.coefs.size(), 0);  // a component no scan coded
        jc.coefs = std::move(c.coefs);
        out.channels.push_back(std::move(jc));
    }
}

}  // namespace

bool decode_jpeg(const uint8_t *data, size_t len, JpegImage &out, std::string &err)
{
    try {
        Decoder dec(data, len);
        dec.run(out);
        return true;
    } catch (const DecodeError &e) {
        err = e.msg;
        return false;
    }
}

}  // namespace art
