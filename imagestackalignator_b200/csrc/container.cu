// DNG container on the host: the TIFF structure RawFile reads
// (PefFile/RawFile.cs:56-90: byte order, magic 42, the IFD chain), SubIFDs
// (IFDSubIFDs, PefFile/ImageFileDirectoryEntry.cs:3794-3860), the raw IFD
// DNGFile.SetMembers picks (PefFile/DNGFile.cs:621-660) and the tags it and
// DNGColorSpec read, turned into the structs of isa_dng_decode,
// isa_dng_levels and isa_dng_color_spec. Every read is bounds-checked; a
// file the reference could not read is ISA_EINVAL.
#include "isa_internal.cuh"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <new>
#include <set>
#include <vector>

namespace {

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return isa_set_error(code, buf);
}

struct Entry {
    uint16_t type = 0;
    uint32_t count = 0;
    size_t at = 0;  // file position of the value bytes (inline in the entry when they fit in 4)
};

struct Ifd {
    std::map<uint16_t, Entry> tags;  // the first entry of a tag wins, as GetEntry returns the first
    const Entry* get(uint16_t t) const
    {
        auto it = tags.find(t);
        return it == tags.end() ? nullptr : &it->second;
    }
};

size_t type_size(uint16_t t)
{
    static const size_t s[14] = {0, 1, 1, 2, 4, 8, 1, 1, 2, 4, 8, 4, 8, 4};  // 13 = IFD offset
    return t < 14 ? s[t] : 0;
}

struct Tiff {
    const uint8_t* d = nullptr;
    size_t n = 0;
    bool big = false;
    bool ok = true;
    long long rel = 0;  // subtracted from out-of-line value offsets (maker notes that store file offsets)
    uint32_t u8(size_t p)
    {
        if (p >= n) { ok = false; return 0; }
        return d[p];
    }
    uint32_t u16(size_t p)
    {
        if (p + 2 > n) { ok = false; return 0; }
        return big ? (uint32_t)d[p] << 8 | d[p + 1] : (uint32_t)d[p + 1] << 8 | d[p];
    }
    uint32_t u32(size_t p)
    {
        if (p + 4 > n) { ok = false; return 0; }
        return big ? (uint32_t)d[p] << 24 | (uint32_t)d[p + 1] << 16 | (uint32_t)d[p + 2] << 8 | d[p + 3]
                   : (uint32_t)d[p + 3] << 24 | (uint32_t)d[p + 2] << 16 | (uint32_t)d[p + 1] << 8 | d[p];
    }
    // one IFD at `o` (ImageFileDirectory): entry count, 12-byte entries; returns the next IFD's offset
    uint32_t ifd(size_t o, Ifd& out)
    {
        const uint32_t cnt = u16(o);
        for (uint32_t i = 0; i < cnt && ok; i++) {
            const size_t e = o + 2 + 12 * (size_t)i;
            Entry en;
            const uint32_t tag = u16(e);
            en.type = (uint16_t)u16(e + 2);
            en.count = u32(e + 4);
            const size_t bytes = type_size(en.type) * (size_t)en.count;
            en.at = bytes <= 4 ? e + 8 : (size_t)((long long)u32(e + 8) - rel);
            if (type_size(en.type) != 0 && en.at + bytes <= n) out.tags.emplace((uint16_t)tag, en);
        }
        return u32(o + 2 + 12 * (size_t)cnt);
    }
    // value i of an entry as a number (rationals as numerator / denominator in double)
    double num(const Entry& e, uint32_t i)
    {
        const size_t s = type_size(e.type), p = e.at + s * i;
        switch (e.type) {
        case 1: case 7: return (double)u8(p);
        case 6: return (double)(int8_t)u8(p);
        case 3: return (double)u16(p);
        case 8: return (double)(int16_t)u16(p);
        case 4: case 13: return (double)u32(p);
        case 9: return (double)(int32_t)u32(p);
        case 5: return (double)u32(p) / (double)u32(p + 4);
        case 10: return (double)(int32_t)u32(p) / (double)(int32_t)u32(p + 4);
        case 11: {
            const uint32_t b = u32(p);
            float f;
            std::memcpy(&f, &b, 4);
            return (double)f;
        }
        case 12: {
            const uint64_t b = (uint64_t)u32(big ? p : p + 4) << 32 | u32(big ? p + 4 : p);
            double v;
            std::memcpy(&v, &b, 8);
            return v;
        }
        default: return 0.0;
        }
    }
    std::vector<double> nums(const Entry* e)
    {
        std::vector<double> v;
        if (!e) return v;
        v.reserve(e->count);
        for (uint32_t i = 0; i < e->count && ok; i++) v.push_back(num(*e, i));
        return v;
    }
};

// TIFF tags read by DNGFile and DNGColorSpec
enum : uint16_t {
    T_WIDTH = 256, T_LENGTH = 257, T_BITS = 258, T_COMPRESSION = 259, T_PHOTOMETRIC = 262, T_STRIP_OFFSETS = 273, T_ROWS_PER_STRIP = 278,
    T_STRIP_BYTES = 279, T_TILE_WIDTH = 322, T_TILE_LENGTH = 323, T_TILE_OFFSETS = 324, T_TILE_BYTES = 325, T_SUBIFDS = 330,
    T_CFA_REPEAT = 33421, T_CFA_PATTERN = 33422, T_EXIF = 34665, T_ISO = 34855, T_DNG_VERSION = 50706, T_CFA_PLANE_COLOR = 50710,
    T_LINEARIZATION = 50712, T_BLACK = 50714, T_BLACK_DH = 50715, T_BLACK_DV = 50716, T_WHITE = 50717, T_CROP_ORIGIN = 50719,
    T_CROP_SIZE = 50720, T_COLOR_MATRIX1 = 50721, T_COLOR_MATRIX2 = 50722, T_CALIBRATION1 = 50723, T_ANALOG_BALANCE = 50727,
    T_AS_SHOT_NEUTRAL = 50728, T_AS_SHOT_WHITE_XY = 50729, T_ILLUMINANT1 = 50778, T_ILLUMINANT2 = 50779, T_ACTIVE_AREA = 50829,
    T_FORWARD_MATRIX1 = 50964, T_FORWARD_MATRIX2 = 50965, T_NOISE_PROFILE = 51041, T_PRIVATE_DATA = 50740,
};
constexpr uint32_t PHOTOMETRIC_CFA = 32803;

}  // namespace

struct isa_dng_file {
    int width = 0, height = 0;
    float roll = 0.f;
    bool roll_present = false;
    std::vector<uint32_t> offsets, counts;
    std::vector<uint16_t> lin;
    std::vector<uint8_t> cfa;
    std::vector<int> plane, active;
    std::vector<double> black, crop_origin, crop_size, noise, dh, dv;
    std::vector<double> cm1, cm2, fm1, fm2, cc1, ab, neutral, white_xy;
    isa_dng_layout layout{};
    isa_dng_level_tags levels{};
    isa_dng_color_tags color{};
};

namespace {

template <class T>
const T* opt(const std::vector<T>& v) { return v.empty() ? nullptr : v.data(); }

// A tag value as an integer of type T, truncated toward zero; NaN and values outside T are refused.
template <class T>
bool as_int(double v, T& out)
{
    if (!(v > (double)std::numeric_limits<T>::min() - 1.0 && v < (double)std::numeric_limits<T>::max() + 1.0)) return false;
    out = (T)v;
    return true;
}

// A Pentax maker note inside `d` (n bytes): PentaxMakerNotes' three headers
// (PefFile/PentaxMakerNotes.cs:26-170). "AOC\0" + byte order: entries at 6,
// value offsets counted from the file's start (`at` = the note's file
// offset); "PENTAX \0" + byte order: entries at 10, offsets from the note's
// start; "Adobe\0MakN" (a DNG's private data) + count + byte order + the
// note's original file offset, then one of the two: offsets moved by the
// 20-byte Adobe header. Returns false for anything else.
bool pentax_note(const uint8_t* d, size_t n, size_t at, Tiff& m, size_t& ifd_at)
{
    m.d = d;
    m.n = n;
    m.ok = true;
    m.rel = 0;
    size_t order = 0;
    if (n >= 6 && std::memcmp(d, "AOC\0", 4) == 0) {
        order = 4;
        ifd_at = 6;
        m.rel = (long long)at;
    } else if (n >= 10 && std::memcmp(d, "PENTAX \0", 8) == 0) {
        order = 8;
        ifd_at = 10;
    } else if (n >= 24 && std::memcmp(d, "Adobe\0MakN", 10) == 0) {
        if (d[14] != d[15] || (d[14] != 'I' && d[14] != 'M')) return false;
        m.big = d[14] == 'M';
        const long long orig = (long long)m.u32(16);
        if (n >= 26 && std::memcmp(d + 20, "AOC\0", 4) == 0) {
            order = 24;
            ifd_at = 26;
            m.rel = orig - 20;
        } else if (n >= 30 && std::memcmp(d + 20, "PENTAX \0", 8) == 0) {
            order = 28;
            ifd_at = 30;
            m.rel = -20;
        } else {
            return false;
        }
    } else {
        return false;
    }
    if (d[order] != d[order + 1] || (d[order] != 'I' && d[order] != 'M')) return false;
    m.big = d[order] == 'M';
    return true;
}

// MNLevelInfo (PefFile/PentaxMakerNotesEntry.cs:4687-4692): the roll angle is -byte 1 / 2 degrees.
constexpr uint16_t MN_LEVEL_INFO = 0x022b;
bool roll_angle(Tiff& m, const Ifd& note, float& deg)
{
    const Entry* e = note.get(MN_LEVEL_INFO);
    if (!e || e->count < 2 || type_size(e->type) != 1) return false;
    deg = (float)(-(int)(int8_t)m.u8(e->at + 1)) / 2.0f;
    return m.ok;
}

#define ISA_TAG_INT(v, out) \
    do { \
        if (!as_int((v), (out))) return fail(ISA_EINVAL, "a tag value is out of range"); \
    } while (0)

int open_dng(const uint8_t* file, size_t size, isa_dng_file& f)
{
    Tiff t;
    t.d = file;
    t.n = size;
    if (size < 8 || file[0] != file[1] || (file[0] != 'I' && file[0] != 'M')) return fail(ISA_EINVAL, "not a TIFF file (byte order)");
    t.big = file[0] == 'M';
    if (t.u16(2) != 42) return fail(ISA_EINVAL, "not a TIFF file (magic number is not 42)");
    // the IFD chain (RawFile.cs:78-88), bounded and without cycles
    std::vector<Ifd> chain;
    std::set<uint32_t> seen;
    for (uint32_t o = t.u32(4); o != 0;) {
        if (!seen.insert(o).second || chain.size() >= 64) return fail(ISA_EINVAL, "IFD chain loops or is too long");
        chain.emplace_back();
        o = t.ifd(o, chain.back());
        if (!t.ok) return fail(ISA_EINVAL, "IFD outside the file");
    }
    if (chain.empty()) return fail(ISA_EINVAL, "no IFD");
    // the raw IFD: the first IFD of the chain with a CFA photometric interpretation, else, for every IFD
    // of the chain in turn, its first CFA SubIFD (a later IFD's replaces an earlier one's; DNGFile.cs:621-660)
    const Ifd* raw = nullptr;
    for (const Ifd& i : chain) {
        const Entry* p = i.get(T_PHOTOMETRIC);
        if (p && t.num(*p, 0) == PHOTOMETRIC_CFA) { raw = &i; break; }
    }
    std::vector<Ifd> subs;
    subs.reserve(64 * 16);
    if (!raw) {
        for (const Ifd& i : chain) {
            const Entry* s = i.get(T_SUBIFDS);
            if (!s) continue;
            for (uint32_t j = 0; j < s->count && j < 16; j++) {
                uint32_t at;
                ISA_TAG_INT(t.num(*s, j), at);
                subs.emplace_back();
                t.ifd(at, subs.back());
                if (!t.ok) return fail(ISA_EINVAL, "SubIFD outside the file");
                const Entry* p = subs.back().get(T_PHOTOMETRIC);
                if (p && t.num(*p, 0) == PHOTOMETRIC_CFA) { raw = &subs.back(); break; }
            }
        }
    }
    if (!raw) return fail(ISA_EINVAL, "no IFD with a CFA image");
    const Ifd& ifd0 = chain[0];
    const auto raw_nums = [&](uint16_t tag) { return t.nums(raw->get(tag)); };
    const auto color_nums = [&](uint16_t tag) {  // DNGColorSpec.GetTag: IFD 0 first, then the raw IFD (DNGColorSpec.cs:94-103)
        const Entry* e = ifd0.get(tag);
        return t.nums(e ? e : raw->get(tag));
    };
    const std::vector<double> w = raw_nums(T_WIDTH), h = raw_nums(T_LENGTH), bits = raw_nums(T_BITS), comp = raw_nums(T_COMPRESSION);
    if (w.empty() || h.empty() || bits.empty() || comp.empty()) return fail(ISA_EINVAL, "raw IFD without size, bit depth or compression");
    ISA_TAG_INT(w[0], f.width);
    ISA_TAG_INT(h[0], f.height);
    const bool tiled = raw->get(T_TILE_WIDTH) != nullptr;
    const std::vector<double> offs = raw_nums(tiled ? T_TILE_OFFSETS : T_STRIP_OFFSETS), cnts = raw_nums(tiled ? T_TILE_BYTES : T_STRIP_BYTES);
    if (offs.empty() || offs.size() != cnts.size()) return fail(ISA_EINVAL, "tile / strip offsets and byte counts do not match");
    for (size_t i = 0; i < offs.size(); i++) {
        uint32_t o, c;
        ISA_TAG_INT(offs[i], o);
        ISA_TAG_INT(cnts[i], c);
        f.offsets.push_back(o);
        f.counts.push_back(c);
    }
    const std::vector<double> lin = raw_nums(T_LINEARIZATION);
    for (double v : lin) {
        uint16_t u;
        ISA_TAG_INT(v, u);
        f.lin.push_back(u);
    }
    const std::vector<double> ver = t.nums(ifd0.get(T_DNG_VERSION));
    isa_dng_layout& L = f.layout;
    L.tiled = tiled ? 1 : 0;
    if (tiled) {
        const std::vector<double> tw = raw_nums(T_TILE_WIDTH), th = raw_nums(T_TILE_LENGTH);
        if (th.empty()) return fail(ISA_EINVAL, "TileWidth without TileLength");
        ISA_TAG_INT(tw[0], L.tile_width);
        ISA_TAG_INT(th[0], L.tile_height);
    } else {
        const std::vector<double> rps = raw_nums(T_ROWS_PER_STRIP);
        L.rows_per_strip = f.height;
        if (!rps.empty()) ISA_TAG_INT(std::min<double>(rps[0], (double)f.height), L.rows_per_strip);
    }
    L.n = (int)f.offsets.size();
    L.offsets = f.offsets.data();
    L.byte_counts = f.counts.data();
    ISA_TAG_INT(comp[0], L.compression);
    ISA_TAG_INT(bits[0], L.bit_depth);
    L.dng_version_large = ver.size() < 2 || ver[1] > 1 ? 1 : 0;  // DNGFile constructor (:288-291)
    L.linearization = opt(f.lin);
    L.nlin = (int)f.lin.size();
    // levels and geometry (DNGFile.SetMembers :706-967 and the constructor :324-372)
    const std::vector<double> rep = raw_nums(T_CFA_REPEAT), pat = raw_nums(T_CFA_PATTERN), white = raw_nums(T_WHITE);
    if (rep.size() < 2 || pat.size() < 4) return fail(ISA_EINVAL, "raw IFD without a CFA pattern");
    if (white.empty()) return fail(ISA_EINVAL, "raw IFD without WhiteLevel");
    for (int i = 0; i < 4; i++) {
        uint8_t c;
        ISA_TAG_INT(pat[i], c);
        f.cfa.push_back(c);
    }
    for (double v : raw_nums(T_CFA_PLANE_COLOR)) {
        int c;
        ISA_TAG_INT(v, c);
        f.plane.push_back(c);
    }
    for (double v : raw_nums(T_ACTIVE_AREA)) {
        int a;
        ISA_TAG_INT(v, a);
        f.active.push_back(a);
    }
    if (!f.active.empty() && f.active.size() != 4) return fail(ISA_EINVAL, "ActiveArea needs four values");
    f.black = raw_nums(T_BLACK);
    f.crop_origin = raw_nums(T_CROP_ORIGIN);
    f.crop_size = raw_nums(T_CROP_SIZE);
    f.noise = raw_nums(T_NOISE_PROFILE);
    if (f.noise.empty()) f.noise = t.nums(ifd0.get(T_NOISE_PROFILE));
    f.dh = raw_nums(T_BLACK_DH);
    f.dv = raw_nums(T_BLACK_DV);
    isa_dng_level_tags& G = f.levels;
    G.width = f.width;
    G.height = f.height;
    G.cfa_pattern = f.cfa.data();
    ISA_TAG_INT(rep[0], G.cfa_repeat_w);
    ISA_TAG_INT(rep[1], G.cfa_repeat_h);
    G.plane_color = opt(f.plane);
    G.n_plane_color = (int)f.plane.size();
    G.black_level = opt(f.black);
    G.n_black = (int)f.black.size();
    G.white_level = white[0];
    G.camera_white = nullptr;  // from isa_dng_color_spec
    G.active_area = opt(f.active);
    G.default_crop_origin = opt(f.crop_origin);
    G.default_crop_size = opt(f.crop_size);
    G.noise_profile = opt(f.noise);
    G.n_noise = (int)f.noise.size();
    G.black_delta_h = opt(f.dh);
    G.n_delta_h = (int)f.dh.size();
    G.black_delta_v = opt(f.dv);
    G.n_delta_v = (int)f.dv.size();
    // ISO: the Exif IFD's ISOSpeedRatings, else the raw IFD's, else IFD 0's (:676-705)
    std::vector<double> iso;
    if (const Entry* ex = ifd0.get(T_EXIF)) {
        Ifd exif;
        uint32_t at;
        ISA_TAG_INT(t.num(*ex, 0), at);
        t.ifd(at, exif);
        if (!t.ok) return fail(ISA_EINVAL, "Exif IFD outside the file");
        iso = t.nums(exif.get(T_ISO));
    } else {
        iso = raw_nums(T_ISO);
        if (iso.empty()) iso = t.nums(ifd0.get(T_ISO));
    }
    G.iso = 0;
    if (!iso.empty()) ISA_TAG_INT(iso[0], G.iso);
    // colour tags (DNGColorSpec.cs:270-392): CameraCalibration1 serves both illuminants, as the reference reads it
    f.cm1 = color_nums(T_COLOR_MATRIX1);
    f.cm2 = color_nums(T_COLOR_MATRIX2);
    f.fm1 = color_nums(T_FORWARD_MATRIX1);
    f.fm2 = color_nums(T_FORWARD_MATRIX2);
    f.cc1 = color_nums(T_CALIBRATION1);
    f.ab = color_nums(T_ANALOG_BALANCE);
    f.neutral = color_nums(T_AS_SHOT_NEUTRAL);
    f.white_xy = color_nums(T_AS_SHOT_WHITE_XY);
    for (const std::vector<double>* m : {&f.cm1, &f.cm2, &f.fm1, &f.fm2, &f.cc1})
        if (!m->empty() && m->size() != 9) return fail(ISA_EINVAL, "a colour matrix of a three-colour camera needs nine values");
    if ((!f.ab.empty() && f.ab.size() != 3) || (!f.neutral.empty() && f.neutral.size() != 3) || (!f.white_xy.empty() && f.white_xy.size() != 2))
        return fail(ISA_EINVAL, "AnalogBalance / AsShotNeutral need three values, AsShotWhiteXY two");
    const std::vector<double> il1 = color_nums(T_ILLUMINANT1), il2 = color_nums(T_ILLUMINANT2);
    isa_dng_color_tags& C = f.color;
    C.color_matrix1 = opt(f.cm1);
    C.color_matrix2 = opt(f.cm2);
    C.illuminant1 = C.illuminant2 = 0;
    if (!il1.empty()) ISA_TAG_INT(il1[0], C.illuminant1);
    if (!il2.empty()) ISA_TAG_INT(il2[0], C.illuminant2);
    C.forward_matrix1 = opt(f.fm1);
    C.forward_matrix2 = opt(f.fm2);
    C.camera_calibration1 = opt(f.cc1);
    C.camera_calibration2 = opt(f.cc1);
    C.analog_balance = opt(f.ab);
    C.as_shot_neutral = opt(f.neutral);
    C.as_shot_white_xy = opt(f.white_xy);
    // the roll angle of a Pentax maker note in DNGPrivateData (DNGFile.cs:676-685)
    if (const Entry* pd = ifd0.get(T_PRIVATE_DATA)) {
        Tiff m;
        size_t ifd_at = 0;
        if (pentax_note(file + pd->at, (size_t)pd->count * type_size(pd->type), pd->at, m, ifd_at)) {
            Ifd note;
            m.ifd(ifd_at, note);
            if (m.ok) f.roll_present = roll_angle(m, note, f.roll);
        }
    }
    if (!t.ok) return fail(ISA_EINVAL, "a tag's values lie outside the file");
    return ISA_OK;
}

}  // namespace

int isa_dng_roll_angle(const isa_dng_file* f, float* roll_deg)
{
    if (!f || !roll_deg) return fail(ISA_EINVAL, "NULL argument");
    *roll_deg = f->roll_present ? f->roll : 0.f;
    return f->roll_present ? 1 : 0;
}

int isa_dng_open(const uint8_t* file, size_t size, isa_dng_file** out)
{
    if (!file || !out) return fail(ISA_EINVAL, "NULL argument");
    *out = nullptr;
    isa_dng_file* f = new (std::nothrow) isa_dng_file();
    if (!f) return fail(ISA_ENOMEM, "out of host memory");
    const int rc = open_dng(file, size, *f);
    if (rc != ISA_OK) {
        delete f;
        return rc;
    }
    *out = f;
    return ISA_OK;
}

int isa_dng_close(isa_dng_file* f)
{
    delete f;
    return ISA_OK;
}

int isa_dng_file_info(const isa_dng_file* f, isa_dng_layout* layout, isa_dng_level_tags* levels, isa_dng_color_tags* color, int* width,
                      int* height)
{
    if (!f) return fail(ISA_EINVAL, "NULL file");
    if (layout) *layout = f->layout;
    if (levels) *levels = f->levels;
    if (color) *color = f->color;
    if (width) *width = f->width;
    if (height) *height = f->height;
    return ISA_OK;
}

// ---- PEF container ----
// PEFFile.SetMembers (PefFile/PEFFile.cs:176-312): the raw image is IFD 0
// (size, bit depth, strips); the Exif IFD holds the ISO, the CFA pattern
// (ExifCFAPattern, PefFile/ExifEntry.cs:2529-2542: repeat counts in bytes 1
// and 3, the colours from byte 4) and the maker note, which PentaxMakerNotes
// (PefFile/PentaxMakerNotes.cs:26-198) reads after an "AOC\0" header (its
// own byte order, entry offsets counted from the file's start) or a
// "PENTAX \0" header (offsets from the maker note's start). The maker-note
// entries used: HuffmanTable 0x0220, BlackPoint 0x0200, WhitePoint 0x0201,
// WhiteLevel 0x007e, DataScaling 0x003d.

struct isa_pef_file {
    std::vector<uint32_t> offsets, sizes;
    std::vector<uint8_t> huff;
    std::vector<float> black;
    isa_pef_info info{};
};

namespace {

enum : uint16_t { T_EXIF_CFA = 41730, T_MAKER_NOTE = 37500, MN_BLACK = 0x0200, MN_WHITE_POINT = 0x0201, MN_WHITE_LEVEL = 0x007e,
                  MN_SCALING = 0x003d, MN_HUFFMAN = 0x0220 };

int open_pef(const uint8_t* file, size_t size, isa_pef_file& f)
{
    Tiff t;
    t.d = file;
    t.n = size;
    if (size < 8 || file[0] != file[1] || (file[0] != 'I' && file[0] != 'M')) return fail(ISA_EINVAL, "not a TIFF file (byte order)");
    t.big = file[0] == 'M';
    if (t.u16(2) != 42) return fail(ISA_EINVAL, "not a TIFF file (magic number is not 42)");
    Ifd raw;
    t.ifd(t.u32(4), raw);
    if (!t.ok) return fail(ISA_EINVAL, "IFD 0 outside the file");
    const std::vector<double> w = t.nums(raw.get(T_WIDTH)), h = t.nums(raw.get(T_LENGTH)), bits = t.nums(raw.get(T_BITS));
    const std::vector<double> offs = t.nums(raw.get(T_STRIP_OFFSETS)), cnts = t.nums(raw.get(T_STRIP_BYTES)), rps = t.nums(raw.get(T_ROWS_PER_STRIP));
    if (w.empty() || h.empty() || bits.empty()) return fail(ISA_EINVAL, "IFD 0 without size or bit depth");
    if (offs.empty() || offs.size() != cnts.size()) return fail(ISA_EINVAL, "strip offsets and byte counts do not match");
    for (size_t i = 0; i < offs.size(); i++) {
        uint32_t o, c;
        ISA_TAG_INT(offs[i], o);
        ISA_TAG_INT(cnts[i], c);
        f.offsets.push_back(o);
        f.sizes.push_back(c);
    }
    const Entry* ex = raw.get(T_EXIF);
    if (!ex) return fail(ISA_EINVAL, "no Exif IFD");
    Ifd exif;
    uint32_t exif_at;
    ISA_TAG_INT(t.num(*ex, 0), exif_at);
    t.ifd(exif_at, exif);
    if (!t.ok) return fail(ISA_EINVAL, "Exif IFD outside the file");
    const Entry* cfa = exif.get(T_EXIF_CFA);
    const Entry* mn = exif.get(T_MAKER_NOTE);
    if (!cfa || cfa->count < 8) return fail(ISA_EINVAL, "no Exif CFA pattern");
    if (!mn) return fail(ISA_EINVAL, "no maker note");
    const uint32_t xc = t.u8(cfa->at + 1), yc = t.u8(cfa->at + 3);
    if (xc != 2 || yc != 2) return fail(ISA_EINVAL, "the CFA pattern is not 2 x 2");
    isa_pef_info& I = f.info;
    for (int i = 0; i < 4; i++) I.cfa[i] = (int)t.u8(cfa->at + 4 + i);
    const std::vector<double> iso = t.nums(exif.get(T_ISO));
    I.iso = 0;
    if (!iso.empty()) ISA_TAG_INT(iso[0], I.iso);
    // the maker note's own byte order and offset base
    const size_t mo = mn->at, mlen = (size_t)mn->count * type_size(mn->type);
    Tiff m;
    size_t ifd_at = 0;
    if (!pentax_note(file + mo, mlen, mo, m, ifd_at)) return fail(ISA_EINVAL, "not a Pentax maker note (header or byte order)");
    Ifd note;
    m.ifd(ifd_at, note);
    if (!m.ok) return fail(ISA_EINVAL, "maker note entries outside the maker note");
    if (const Entry* hu = note.get(MN_HUFFMAN)) {
        const size_t nb = (size_t)hu->count * type_size(hu->type);
        f.huff.assign(m.d + hu->at, m.d + hu->at + nb);
    }
    for (double v : m.nums(note.get(MN_BLACK))) f.black.push_back((float)v);
    const std::vector<double> wp = m.nums(note.get(MN_WHITE_POINT)), wl = m.nums(note.get(MN_WHITE_LEVEL)), sc = m.nums(note.get(MN_SCALING));
    if (wp.size() < 4 || sc.empty()) return fail(ISA_EINVAL, "maker note without WhitePoint or DataScaling");
    ISA_TAG_INT(w[0], I.width);
    ISA_TAG_INT(h[0], I.height);
    ISA_TAG_INT(bits[0], I.bit_depth);
    I.nstrips = (int)f.offsets.size();
    I.strip_offsets = f.offsets.data();
    I.strip_sizes = f.sizes.data();
    I.rows_per_strip = I.height;
    if (!rps.empty()) ISA_TAG_INT(std::min<double>(rps[0], (double)I.height), I.rows_per_strip);
    I.compressed = !f.huff.empty() && I.nstrips == 1 ? 1 : 0;  // PEFFile.cs:87
    I.huffman_table = opt(f.huff);
    I.huffman_bytes = f.huff.size();
    I.huffman_big_endian = m.big ? 1 : 0;
    I.black_point = opt(f.black);
    I.n_black = (int)f.black.size();
    I.white_level = wl.empty() ? -1.f : (float)wl[0];
    for (int i = 0; i < 4; i++) I.white_point[i] = (float)wp[i];
    I.scaling = (float)sc[0];
    I.roll_angle = 0.f;
    I.roll_angle_present = roll_angle(m, note, I.roll_angle) ? 1 : 0;
    if (!t.ok || !m.ok) return fail(ISA_EINVAL, "a tag's values lie outside the file");
    return ISA_OK;
}

}  // namespace

int isa_pef_open(const uint8_t* file, size_t size, isa_pef_file** out)
{
    if (!file || !out) return fail(ISA_EINVAL, "NULL argument");
    *out = nullptr;
    isa_pef_file* f = new (std::nothrow) isa_pef_file();
    if (!f) return fail(ISA_ENOMEM, "out of host memory");
    const int rc = open_pef(file, size, *f);
    if (rc != ISA_OK) {
        delete f;
        return rc;
    }
    *out = f;
    return ISA_OK;
}

int isa_pef_close(isa_pef_file* f)
{
    delete f;
    return ISA_OK;
}

int isa_pef_file_info(const isa_pef_file* f, isa_pef_info* info)
{
    if (!f || !info) return fail(ISA_EINVAL, "NULL argument");
    *info = f->info;
    return ISA_OK;
}
