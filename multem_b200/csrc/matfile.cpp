// Level-5 MAT-file reader and writer (format summary in matfile.hpp).
#include "matfile.hpp"

#include <zlib.h>

#include <cstring>
#include <ctime>
#include <fstream>
#include <iterator>

#include "common.hpp"

namespace mtb {
namespace mat {
namespace {

enum DataType : uint32_t {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6, miSINGLE = 7,
    miDOUBLE = 9, miINT64 = 12, miUINT64 = 13, miMATRIX = 14, miCOMPRESSED = 15, miUTF8 = 16,
    miUTF16 = 17, miUTF32 = 18
};

constexpr uint32_t kFlagComplex = 0x0800, kFlagLogical = 0x0200;

[[noreturn]] void bad(const std::string& what) { fail(MT_ERR_INVALID_ARG, "MAT-file: " + what); }

uint32_t u32(const uint8_t* p) {
    uint32_t v;
    std::memcpy(&v, p, 4);
    return v;
}

size_t pad8(size_t n) { return (n + 7) & ~size_t(7); }

// One data element inside [p, end): its type, data and the bytes it occupies (tag + padded data).
struct Element {
    uint32_t type = 0;
    const uint8_t* data = nullptr;
    size_t nbytes = 0;
    size_t span = 0;
};

Element next_element(const uint8_t* p, const uint8_t* end, bool pad) {
    if (end - p < 8) bad("truncated data element tag");
    Element e;
    const uint32_t first = u32(p);
    if (first >> 16) {  // small data element: 2-byte count, 2-byte type, data in the next 4 bytes
        e.type = first & 0xFFFF;
        e.nbytes = first >> 16;
        if (e.nbytes > 4) bad("small data element longer than 4 bytes");
        e.data = p + 4;
        e.span = 8;
        return e;
    }
    e.type = first;
    e.nbytes = u32(p + 4);
    e.data = p + 8;
    e.span = 8 + (pad ? pad8(e.nbytes) : e.nbytes);
    if ((size_t)(end - e.data) < e.nbytes) bad("data element runs past the end of its container");
    if ((size_t)(end - p) < e.span) e.span = (size_t)(end - p);  // last element, padding omitted
    return e;
}

template <class T>
void append_as(const uint8_t* d, size_t nbytes, std::vector<double>& out) {
    const size_t n = nbytes / sizeof(T);
    out.reserve(out.size() + n);
    for (size_t i = 0; i < n; i++) {
        T v;
        std::memcpy(&v, d + i * sizeof(T), sizeof(T));
        out.push_back((double)v);
    }
}

// Numeric (or character) data of any storage type, as doubles.
std::vector<double> numeric(const Element& e) {
    std::vector<double> v;
    switch (e.type) {
        case miINT8: append_as<int8_t>(e.data, e.nbytes, v); break;
        case miUINT8: append_as<uint8_t>(e.data, e.nbytes, v); break;
        case miINT16: append_as<int16_t>(e.data, e.nbytes, v); break;
        case miUINT16: append_as<uint16_t>(e.data, e.nbytes, v); break;
        case miUTF16: append_as<uint16_t>(e.data, e.nbytes, v); break;
        case miINT32: append_as<int32_t>(e.data, e.nbytes, v); break;
        case miUINT32: append_as<uint32_t>(e.data, e.nbytes, v); break;
        case miUTF32: append_as<uint32_t>(e.data, e.nbytes, v); break;
        case miSINGLE: append_as<float>(e.data, e.nbytes, v); break;
        case miDOUBLE: append_as<double>(e.data, e.nbytes, v); break;
        case miINT64: append_as<int64_t>(e.data, e.nbytes, v); break;
        case miUINT64: append_as<uint64_t>(e.data, e.nbytes, v); break;
        case miUTF8: {  // decode to code points
            for (size_t i = 0; i < e.nbytes;) {
                const uint8_t c = e.data[i];
                int len = c < 0x80 ? 1 : (c >> 5) == 6 ? 2 : (c >> 4) == 14 ? 3 : 4;
                uint32_t cp = len == 1 ? c : len == 2 ? (c & 0x1F) : len == 3 ? (c & 0x0F) : (c & 0x07);
                for (int k = 1; k < len && i + k < e.nbytes; k++) cp = (cp << 6) | (e.data[i + k] & 0x3F);
                v.push_back((double)cp);
                i += len;
            }
            break;
        }
        default: bad("unsupported numeric data type " + std::to_string(e.type));
    }
    return v;
}

Value parse_matrix(const uint8_t* p, size_t n, std::string* name);

// An miMATRIX element nested in a struct or cell (empty when its byte count is 0).
Value parse_nested(const uint8_t*& p, const uint8_t* end) {
    Element e = next_element(p, end, true);
    if (e.type != miMATRIX) bad("struct or cell element is not a matrix");
    Value v;
    if (e.nbytes > 0) v = parse_matrix(e.data, e.nbytes, nullptr);
    p += e.span;
    return v;
}

Value parse_matrix(const uint8_t* p, size_t n, std::string* name) {
    const uint8_t* end = p + n;
    Value v;
    Element flags = next_element(p, end, true);
    if (flags.type != miUINT32 || flags.nbytes < 8) bad("missing array flags");
    const uint32_t f = u32(flags.data);
    v.cls = (int)(f & 0xFF);
    v.complex = (f & kFlagComplex) != 0;
    v.logical = (f & kFlagLogical) != 0;
    p += flags.span;
    Element dims = next_element(p, end, true);
    if (dims.type != miINT32 || dims.nbytes < 8) bad("missing dimensions");
    v.dims.clear();
    for (size_t i = 0; i < dims.nbytes / 4; i++) v.dims.push_back((int32_t)u32(dims.data + 4 * i));
    p += dims.span;
    Element nm = next_element(p, end, true);
    if (nm.type != miINT8 && nm.type != miUINT8 && nm.type != miUTF8) bad("missing array name");
    if (name) name->assign(reinterpret_cast<const char*>(nm.data), nm.nbytes);
    p += nm.span;
    const size_t count = v.numel();
    switch (v.cls) {
        case kStruct: {
            Element fl = next_element(p, end, true);
            if (fl.type != miINT32 || fl.nbytes != 4) bad("missing struct field-name length");
            const size_t len = u32(fl.data);
            p += fl.span;
            Element fn = next_element(p, end, true);
            if (fn.type != miINT8 && fn.type != miUINT8) bad("missing struct field names");
            if (len == 0 || fn.nbytes % len) bad("malformed struct field names");
            for (size_t i = 0; i < fn.nbytes / len; i++) {
                const char* s = reinterpret_cast<const char*>(fn.data + i * len);
                v.fields.emplace_back(s, strnlen(s, len));
            }
            p += fn.span;
            for (size_t i = 0; i < count * v.fields.size(); i++) v.elems.push_back(parse_nested(p, end));
            break;
        }
        case kCell:
            for (size_t i = 0; i < count; i++) v.elems.push_back(parse_nested(p, end));
            break;
        case kObject: bad("objects are not supported (save the struct from toStruct)");
        case kSparse: bad("sparse arrays are not supported");
        default: {
            if (v.cls < kChar || v.cls > kUInt64) bad("unknown array class " + std::to_string(v.cls));
            if (count == 0) break;
            Element re = next_element(p, end, true);
            v.re = numeric(re);
            p += re.span;
            if (v.complex) {
                Element im = next_element(p, end, true);
                v.im = numeric(im);
                p += im.span;
            }
            if (v.re.size() != count || (v.complex && v.im.size() != count)) bad("array data do not match its dimensions");
        }
    }
    return v;
}

std::vector<uint8_t> inflate_all(const uint8_t* p, size_t n) {
    std::vector<uint8_t> out(n * 4 + 1024);
    z_stream zs{};
    if (inflateInit(&zs) != Z_OK) bad("zlib initialisation failed");
    zs.next_in = const_cast<Bytef*>(p);
    zs.avail_in = (uInt)n;
    int r = Z_OK;
    while (true) {
        zs.next_out = out.data() + zs.total_out;
        zs.avail_out = (uInt)(out.size() - zs.total_out);
        r = inflate(&zs, Z_NO_FLUSH);
        if (r == Z_STREAM_END) break;
        if (r != Z_OK && r != Z_BUF_ERROR) {
            inflateEnd(&zs);
            bad("corrupt compressed variable");
        }
        if (zs.avail_out == 0) out.resize(out.size() * 2);
        else if (zs.avail_in == 0) break;  // input exhausted (MATLAB streams end cleanly)
    }
    out.resize(zs.total_out);
    inflateEnd(&zs);
    return out;
}

// ---- writer

struct Out {
    std::vector<uint8_t> b;
    void raw(const void* p, size_t n) {
        const uint8_t* q = static_cast<const uint8_t*>(p);
        b.insert(b.end(), q, q + n);
    }
    void u32v(uint32_t v) { raw(&v, 4); }
    void pad() { b.resize(pad8(b.size()), 0); }
    // a full data element (tag + data + padding)
    void element(uint32_t type, const void* p, size_t n) {
        if (n > 0x7FFFFFFFu) bad("variable larger than the 2^31-byte limit of level-5 MAT-files");
        u32v(type);
        u32v((uint32_t)n);
        raw(p, n);
        pad();
    }
};

void write_matrix(Out& o, const std::string& name, const Value& v) {
    Out m;
    const uint32_t flags = (uint32_t)v.cls | (v.complex ? kFlagComplex : 0) | (v.logical ? kFlagLogical : 0);
    const uint32_t af[2] = {flags, 0};
    m.element(miUINT32, af, 8);
    std::vector<int32_t> d(v.dims.begin(), v.dims.end());
    m.element(miINT32, d.data(), d.size() * 4);
    m.element(miINT8, name.data(), name.size());
    if (v.cls == kStruct) {
        size_t len = 1;
        for (auto& f : v.fields) len = std::max(len, f.size() + 1);
        if (len > 64) bad("struct field name longer than 63 characters");
        const int32_t L = (int32_t)len;
        // field-name length as a small data element
        m.u32v((4u << 16) | miINT32);
        m.raw(&L, 4);
        std::vector<char> names(len * v.fields.size(), 0);
        for (size_t i = 0; i < v.fields.size(); i++) std::memcpy(&names[i * len], v.fields[i].data(), v.fields[i].size());
        m.element(miINT8, names.data(), names.size());
        for (auto& e : v.elems) write_matrix(m, "", e);
    } else if (v.cls == kCell) {
        for (auto& e : v.elems) write_matrix(m, "", e);
    } else if (v.cls == kChar) {
        std::vector<uint16_t> c(v.re.begin(), v.re.end());
        m.element(miUTF16, c.data(), c.size() * 2);
    } else {
        if (v.cls != kDouble) bad("the writer stores double, char, struct and cell arrays only");
        m.element(miDOUBLE, v.re.data(), v.re.size() * 8);
        if (v.complex) m.element(miDOUBLE, v.im.data(), v.im.size() * 8);
    }
    o.element(miMATRIX, m.b.data(), m.b.size());
}

}  // namespace

size_t Value::numel() const {
    size_t n = 1;
    for (auto d : dims) n *= (size_t)(d < 0 ? 0 : d);
    return n;
}

const Value* Value::field(const std::string& name, size_t e) const {
    if (cls != kStruct) return nullptr;
    for (size_t f = 0; f < fields.size(); f++)
        if (fields[f] == name) {
            const size_t i = e * fields.size() + f;
            return i < elems.size() ? &elems[i] : nullptr;
        }
    return nullptr;
}

std::string Value::str() const {
    std::string s;
    for (double c : re) s.push_back((char)(int)c);
    return s;
}

Value Value::scalar(double x) {
    Value v;
    v.dims = {1, 1};
    v.re = {x};
    return v;
}

Value Value::row(const std::vector<double>& x) {
    Value v;
    v.dims = {1, (int64_t)x.size()};
    v.re = x;
    return v;
}

Value Value::matrix(int64_t rows, int64_t cols, const double* re, const double* im, size_t im_stride) {
    Value v;
    v.dims = {rows, cols};
    const size_t n = (size_t)(rows * cols);
    if (im) {
        // interleaved (re, im) pairs when im_stride is 2 (re then points at the first real part)
        v.complex = true;
        v.re.resize(n);
        v.im.resize(n);
        for (size_t i = 0; i < n; i++) {
            v.re[i] = re[i * im_stride];
            v.im[i] = im[i * im_stride];
        }
    } else {
        v.re.assign(re, re + n);
    }
    return v;
}

Value Value::string(const std::string& s) {
    Value v;
    v.cls = kChar;
    v.dims = {1, (int64_t)s.size()};
    for (char c : s) v.re.push_back((double)(unsigned char)c);
    return v;
}

Value Value::struct_array(int64_t rows, int64_t cols, std::vector<std::string> f) {
    Value v;
    v.cls = kStruct;
    v.dims = {rows, cols};
    v.fields = std::move(f);
    v.elems.resize((size_t)(rows * cols) * v.fields.size());
    return v;
}

Value& Value::at(size_t e, const std::string& name) {
    for (size_t f = 0; f < fields.size(); f++)
        if (fields[f] == name) return elems[e * fields.size() + f];
    bad("no struct field " + name);
}

Variables read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) bad("cannot open " + path);
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (buf.size() < 128) bad(path + " is too short for a MAT-file header");
    if (buf[126] == 'M' && buf[127] == 'I') bad("big-endian MAT-files are not supported");
    if (!(buf[126] == 'I' && buf[127] == 'M')) {
        if (buf.size() >= 512 && std::memcmp(buf.data() + 512, "\x89HDF", 4) == 0)
            bad("-v7.3 (HDF5) MAT-files are not supported; save with -v7");
        bad(path + " is not a level-5 MAT-file");
    }
    Variables vars;
    const uint8_t* p = buf.data() + 128;
    const uint8_t* end = buf.data() + buf.size();
    while (end - p >= 8) {
        Element e = next_element(p, end, false);
        std::vector<uint8_t> inflated;
        const uint8_t* mp = e.data;
        size_t mn = e.nbytes;
        if (e.type == miCOMPRESSED) {
            inflated = inflate_all(e.data, e.nbytes);
            const uint8_t* ip = inflated.data();
            Element inner = next_element(ip, ip + inflated.size(), true);
            if (inner.type != miMATRIX) bad("compressed element does not hold a variable");
            mp = inner.data;
            mn = inner.nbytes;
        } else if (e.type != miMATRIX) {
            p += pad8(e.nbytes) + 8;  // not a variable (e.g. subsystem data): skip
            continue;
        }
        std::string name;
        Value v = parse_matrix(mp, mn, &name);
        vars.emplace_back(name, std::move(v));
        p += e.type == miCOMPRESSED ? e.span : pad8(e.nbytes) + 8;
    }
    return vars;
}

void write_file(const std::string& path, const Variables& vars, bool compress) {
    Out o;
    char hdr[128];
    std::memset(hdr, ' ', sizeof(hdr));
    const std::time_t now = std::time(nullptr);
    char when[64];
    std::strftime(when, sizeof(when), "%a %b %d %H:%M:%S %Y", std::gmtime(&now));
    const std::string text = std::string("MATLAB 5.0 MAT-file, Platform: GLNXA64, Created on: ") + when + " by multem_b200";
    std::memcpy(hdr, text.data(), std::min(text.size(), (size_t)116));
    std::memset(hdr + 116, 0, 8);  // no subsystem data
    const uint16_t version = 0x0100;
    std::memcpy(hdr + 124, &version, 2);
    hdr[126] = 'I';
    hdr[127] = 'M';
    o.raw(hdr, 128);
    for (auto& [name, v] : vars) {
        Out m;
        write_matrix(m, name, v);
        if (!compress) {
            o.raw(m.b.data(), m.b.size());
            continue;
        }
        uLongf zn = compressBound((uLong)m.b.size());
        std::vector<uint8_t> z(zn);
        if (compress2(z.data(), &zn, m.b.data(), (uLong)m.b.size(), Z_DEFAULT_COMPRESSION) != Z_OK)
            bad("zlib compression failed");
        if (zn > 0x7FFFFFFFu) bad("variable larger than the 2^31-byte limit of level-5 MAT-files");
        o.u32v(miCOMPRESSED);
        o.u32v((uint32_t)zn);
        o.raw(z.data(), zn);
    }
    std::ofstream out(path, std::ios::binary | std::ios::trunc);
    if (!out) bad("cannot create " + path);
    out.write(reinterpret_cast<const char*>(o.b.data()), (std::streamsize)o.b.size());
    if (!out) bad("cannot write " + path);
}

}  // namespace mat
}  // namespace mtb
