// Minimal NumPy .npz reader/writer for the euler2d host driver.
//
// The reference driver stores snapshots, initial conditions and trajectories as HDF5 datasets with
// attributes (solver/src/io_hdf5.hpp:56-206, solver/src/trajectory.hpp:53-91).  libhdf5 is not
// available to this build, so the driver keeps the same dataset and attribute names and shapes but
// writes them as one .npz archive per file: every dataset is a .npy member, every attribute a 0-d
// .npy member (float64, int32 or a unicode string).  numpy.load() reads the result directly.
//
// Writer: ZIP "stored" members (no compression), ZIP64 not needed below 4 GiB per archive.
// Reader: stored members as numpy.savez writes them (ZIP64 extra fields understood); compressed
// archives (numpy.savez_compressed) are rejected with a clear message.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace npz {

// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320), the checksum ZIP members carry.
inline uint32_t crc32(const unsigned char* p, size_t n, uint32_t crc = 0) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t k = 0; k < 256; ++k) {
            uint32_t c = k;
            for (int b = 0; b < 8; ++b) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
            table[k] = c;
        }
        init = true;
    }
    crc = ~crc;
    for (size_t k = 0; k < n; ++k) crc = table[(crc ^ p[k]) & 0xFFu] ^ (crc >> 8);
    return ~crc;
}

struct Array {
    std::string descr;            // numpy dtype string: "<f8", "<f4", "<i4", "<i8", "<U12", ...
    std::vector<size_t> shape;    // empty for a 0-d array
    std::vector<unsigned char> data;

    size_t count() const {
        size_t n = 1;
        for (size_t s : shape) n *= s;
        return n;
    }
    double scalar() const {       // a 0-d (or 1-element) numeric array as double
        if (count() != 1) throw std::runtime_error("expected a scalar");
        if (descr == "<f8") { double v; std::memcpy(&v, data.data(), 8); return v; }
        if (descr == "<f4") { float v; std::memcpy(&v, data.data(), 4); return v; }
        if (descr == "<i8") { int64_t v; std::memcpy(&v, data.data(), 8); return double(v); }
        if (descr == "<i4") { int32_t v; std::memcpy(&v, data.data(), 4); return double(v); }
        throw std::runtime_error("scalar of unsupported dtype " + descr);
    }
    std::string str() const {     // a unicode string array ("<U<n>", UTF-32LE) with ASCII content
        if (descr.size() < 3 || descr[1] != 'U') throw std::runtime_error("expected a string, got " + descr);
        std::string s;
        for (size_t k = 0; k + 4 <= data.size(); k += 4) {
            uint32_t c;
            std::memcpy(&c, data.data() + k, 4);
            if (c == 0) break;
            s.push_back(c < 128 ? char(c) : '?');
        }
        return s;
    }
    std::vector<double> doubles() const {  // any supported numeric dtype, converted
        std::vector<double> v(count());
        for (size_t k = 0; k < v.size(); ++k) {
            if (descr == "<f8") std::memcpy(&v[k], data.data() + 8 * k, 8);
            else if (descr == "<f4") { float f; std::memcpy(&f, data.data() + 4 * k, 4); v[k] = f; }
            else if (descr == "<i8") { int64_t x; std::memcpy(&x, data.data() + 8 * k, 8); v[k] = double(x); }
            else if (descr == "<i4") { int32_t x; std::memcpy(&x, data.data() + 4 * k, 4); v[k] = double(x); }
            else throw std::runtime_error("array of unsupported dtype " + descr);
        }
        return v;
    }
};

inline Array f64(const std::vector<size_t>& shape, const double* p) {
    Array a{"<f8", shape, {}};
    a.data.resize(a.count() * 8);
    std::memcpy(a.data.data(), p, a.data.size());
    return a;
}
inline Array f32(const std::vector<size_t>& shape, const float* p) {
    Array a{"<f4", shape, {}};
    a.data.resize(a.count() * 4);
    std::memcpy(a.data.data(), p, a.data.size());
    return a;
}
inline Array scalar(double v) { return f64({}, &v); }
inline Array scalar_int(int32_t v) {
    Array a{"<i4", {}, std::vector<unsigned char>(4)};
    std::memcpy(a.data.data(), &v, 4);
    return a;
}
inline Array string(const std::string& s) {
    const size_t n = s.empty() ? 1 : s.size();
    Array a{"<U" + std::to_string(n), {}, std::vector<unsigned char>(4 * n, 0)};
    for (size_t k = 0; k < s.size(); ++k) a.data[4 * k] = (unsigned char)s[k];
    return a;
}

// The .npy v1.0 encoding of one array: magic, header dict padded so the data start on a 64-byte
// boundary, then the raw little-endian C-order data.
inline std::vector<unsigned char> npy_bytes(const Array& a) {
    std::string shape = "(";
    for (size_t k = 0; k < a.shape.size(); ++k) shape += std::to_string(a.shape[k]) + (a.shape.size() == 1 ? "," : (k + 1 < a.shape.size() ? ", " : ""));
    shape += ")";
    std::string h = "{'descr': '" + a.descr + "', 'fortran_order': False, 'shape': " + shape + ", }";
    const size_t pre = 10;
    size_t total = pre + h.size() + 1;
    h.append((64 - total % 64) % 64, ' ');
    h.push_back('\n');
    std::vector<unsigned char> out;
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    out.insert(out.end(), magic, magic + 8);
    out.push_back((unsigned char)(h.size() & 0xFF));
    out.push_back((unsigned char)(h.size() >> 8));
    out.insert(out.end(), h.begin(), h.end());
    out.insert(out.end(), a.data.begin(), a.data.end());
    return out;
}

inline void put16(std::vector<unsigned char>& b, uint16_t v) { b.push_back(v & 0xFF); b.push_back(v >> 8); }
inline void put32(std::vector<unsigned char>& b, uint32_t v) { for (int k = 0; k < 4; ++k) b.push_back((v >> (8 * k)) & 0xFF); }

// Writes name -> array members (".npy" appended to each name) as one stored ZIP archive; the file
// appears complete or not at all (written to path + ".tmp", then renamed).
inline void write(const std::string& path, const std::vector<std::pair<std::string, Array>>& members) {
    std::vector<unsigned char> central;
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) throw std::runtime_error("could not create " + path + " (does the folder exist?)");
    uint64_t offset = 0;
    for (const auto& m : members) {
        const std::string name = m.first + ".npy";
        const std::vector<unsigned char> body = npy_bytes(m.second);
        if (body.size() >= 0xFFFFFFFFull || offset >= 0xFFFFFFFFull) {
            std::fclose(f);
            std::remove(tmp.c_str());
            throw std::runtime_error("archive member " + name + " exceeds 4 GiB");
        }
        const uint32_t crc = crc32(body.data(), body.size());
        std::vector<unsigned char> hdr;
        put32(hdr, 0x04034b50u); put16(hdr, 20); put16(hdr, 0); put16(hdr, 0); put16(hdr, 0); put16(hdr, 0x21);
        put32(hdr, crc); put32(hdr, uint32_t(body.size())); put32(hdr, uint32_t(body.size()));
        put16(hdr, uint16_t(name.size())); put16(hdr, 0);
        hdr.insert(hdr.end(), name.begin(), name.end());
        std::fwrite(hdr.data(), 1, hdr.size(), f);
        std::fwrite(body.data(), 1, body.size(), f);
        put32(central, 0x02014b50u); put16(central, 20); put16(central, 20); put16(central, 0); put16(central, 0);
        put16(central, 0); put16(central, 0x21); put32(central, crc); put32(central, uint32_t(body.size()));
        put32(central, uint32_t(body.size())); put16(central, uint16_t(name.size())); put16(central, 0);
        put16(central, 0); put16(central, 0); put16(central, 0); put32(central, 0); put32(central, uint32_t(offset));
        central.insert(central.end(), name.begin(), name.end());
        offset += hdr.size() + body.size();
    }
    std::vector<unsigned char> end;
    put32(end, 0x06054b50u); put16(end, 0); put16(end, 0); put16(end, uint16_t(members.size()));
    put16(end, uint16_t(members.size())); put32(end, uint32_t(central.size())); put32(end, uint32_t(offset));
    put16(end, 0);
    std::fwrite(central.data(), 1, central.size(), f);
    std::fwrite(end.data(), 1, end.size(), f);
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) {
        std::remove(tmp.c_str());
        throw std::runtime_error("could not write " + path);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("could not create " + path);
}

namespace detail {
inline uint16_t get16(const unsigned char* p) { return uint16_t(p[0] | (p[1] << 8)); }
inline uint32_t get32(const unsigned char* p) { return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24); }
inline uint64_t get64(const unsigned char* p) { return uint64_t(get32(p)) | (uint64_t(get32(p + 4)) << 32); }

inline Array parse_npy(const unsigned char* p, size_t n, const std::string& name) {
    if (n < 10 || std::memcmp(p, "\x93NUMPY", 6) != 0) throw std::runtime_error(name + " is not a .npy array");
    size_t hl, pre;
    if (p[6] == 1) { hl = get16(p + 8); pre = 10; }
    else { hl = get32(p + 8); pre = 12; }
    if (pre + hl > n) throw std::runtime_error(name + ": truncated .npy header");
    const std::string h(reinterpret_cast<const char*>(p + pre), hl);
    auto field = [&](const std::string& key) {
        size_t k = h.find("'" + key + "'");
        if (k == std::string::npos) throw std::runtime_error(name + ": .npy header lacks " + key);
        k = h.find(':', k) + 1;
        while (k < h.size() && h[k] == ' ') ++k;
        return k;
    };
    Array a;
    size_t k = field("descr");
    const char q = h[k];
    a.descr = h.substr(k + 1, h.find(q, k + 1) - k - 1);
    if (a.descr[0] == '|' && a.descr.size() == 3 && a.descr[1] == 'u' && a.descr[2] == '1') a.descr = "|u1";
    k = field("fortran_order");
    if (h.compare(k, 4, "True") == 0) throw std::runtime_error(name + ": Fortran-ordered arrays are not supported");
    k = field("shape");
    const size_t e = h.find(')', k);
    std::string dims = h.substr(k + 1, e - k - 1);
    for (size_t s = 0; s < dims.size();) {
        while (s < dims.size() && (dims[s] == ' ' || dims[s] == ',')) ++s;
        if (s >= dims.size()) break;
        size_t t = s;
        while (t < dims.size() && dims[t] >= '0' && dims[t] <= '9') ++t;
        if (t == s) throw std::runtime_error(name + ": bad shape in .npy header");
        a.shape.push_back(std::stoull(dims.substr(s, t - s)));
        s = t;
    }
    size_t item;
    if (a.descr[1] == 'U') item = 4 * std::stoull(a.descr.substr(2));
    else if (a.descr == "<f8" || a.descr == "<i8") item = 8;
    else if (a.descr == "<f4" || a.descr == "<i4") item = 4;
    else throw std::runtime_error(name + ": unsupported dtype " + a.descr);
    const size_t bytes = a.count() * item;
    if (pre + hl + bytes > n) throw std::runtime_error(name + ": truncated .npy data");
    a.data.assign(p + pre + hl, p + pre + hl + bytes);
    return a;
}
}  // namespace detail

// Reads every .npy member of an archive written by numpy.savez (or by write() above).
inline std::map<std::string, Array> read(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("could not open " + path + " (does the file exist?)");
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    std::fclose(f);
    using namespace detail;
    if (buf.size() < 22) throw std::runtime_error(path + " is not an .npz archive");
    size_t eocd = std::string::npos;
    for (size_t k = buf.size() - 22 + 1; k-- > 0 && buf.size() - k <= 22 + 65535;)
        if (get32(&buf[k]) == 0x06054b50u) { eocd = k; break; }
    if (eocd == std::string::npos) throw std::runtime_error(path + " is not an .npz archive");
    uint64_t entries = get16(&buf[eocd + 10]);
    uint64_t cd = get32(&buf[eocd + 16]);
    if ((cd == 0xFFFFFFFFu || entries == 0xFFFF) && eocd >= 20 && get32(&buf[eocd - 20]) == 0x07064b50u) {
        const uint64_t z = get64(&buf[eocd - 20 + 8]);
        if (z + 56 > buf.size() || get32(&buf[z]) != 0x06064b50u) throw std::runtime_error(path + ": bad ZIP64 record");
        entries = get64(&buf[z + 32]);
        cd = get64(&buf[z + 48]);
    }
    std::map<std::string, Array> out;
    size_t p = cd;
    for (uint64_t e = 0; e < entries; ++e) {
        if (p + 46 > buf.size() || get32(&buf[p]) != 0x02014b50u) throw std::runtime_error(path + ": bad central directory");
        const uint16_t method = get16(&buf[p + 10]);
        uint64_t csize = get32(&buf[p + 20]), usize = get32(&buf[p + 24]);
        const uint16_t nl = get16(&buf[p + 28]), xl = get16(&buf[p + 30]), cl = get16(&buf[p + 32]);
        uint64_t off = get32(&buf[p + 42]);
        std::string name(reinterpret_cast<const char*>(&buf[p + 46]), nl);
        for (size_t x = p + 46 + nl; x + 4 <= p + 46 + nl + xl;) {  // ZIP64 extra: the 0xFFFFFFFF fields, in order
            const uint16_t id = get16(&buf[x]), sz = get16(&buf[x + 2]);
            if (id == 0x0001) {
                size_t q = x + 4;
                if (usize == 0xFFFFFFFFu) { usize = get64(&buf[q]); q += 8; }
                if (csize == 0xFFFFFFFFu) { csize = get64(&buf[q]); q += 8; }
                if (off == 0xFFFFFFFFu) { off = get64(&buf[q]); q += 8; }
            }
            x += 4 + sz;
        }
        p += 46 + nl + xl + cl;
        if (method != 0)
            throw std::runtime_error(path + ": member " + name + " is compressed; write the file with numpy.savez");
        if (off + 30 > buf.size() || get32(&buf[off]) != 0x04034b50u) throw std::runtime_error(path + ": bad member header");
        const size_t data = off + 30 + get16(&buf[off + 26]) + get16(&buf[off + 28]);
        if (data + usize > buf.size()) throw std::runtime_error(path + ": truncated member " + name);
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".npy") == 0) name.resize(name.size() - 4);
        out[name] = parse_npy(&buf[data], usize, name);
    }
    return out;
}

}  // namespace npz
