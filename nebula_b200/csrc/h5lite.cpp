// HDF5-subset reader; see h5lite.h for the supported structures.
#include "h5lite.h"

#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace nbx {
namespace h5 {

namespace {
const uint8_t kSignature[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};

std::vector<std::string> split_path(const std::string& path) {
    std::vector<std::string> parts;
    std::string cur;
    for (char c : path) {
        if (c == '/') {
            if (!cur.empty()) parts.push_back(cur);
            cur.clear();
        } else {
            cur.push_back(c);
        }
    }
    if (!cur.empty()) parts.push_back(cur);
    return parts;
}

[[noreturn]] void fail(const std::string& file, const std::string& what) {
    throw std::runtime_error("HDF5 file " + file + ": " + what);
}
}  // namespace

File::File(const std::string& filename) : filename_(filename) {
    std::ifstream ifs(filename, std::ios::binary);
    if (!ifs.is_open()) throw std::runtime_error("Unable to open file " + filename);
    buf_.assign(std::istreambuf_iterator<char>(ifs), std::istreambuf_iterator<char>());

    // The superblock may follow a user block of 512, 1024, 2048, ... bytes.
    uint64_t sb = UINT64_MAX;
    for (uint64_t off = 0; off + 8 <= buf_.size(); off = (off == 0 ? 512 : off * 2)) {
        if (std::memcmp(buf_.data() + off, kSignature, 8) == 0) {
            sb = off;
            break;
        }
    }
    if (sb == UINT64_MAX) fail(filename_, "no HDF5 signature");
    need(sb, 16);
    const int version = buf_[sb + 8];
    if (version == 0 || version == 1) {
        sizeof_addr_ = buf_[sb + 13];
        sizeof_len_ = buf_[sb + 14];
        uint64_t p = sb + 24 + (version == 1 ? 4 : 0);
        base_ = rd(p, sizeof_addr_);
        p += 4 * sizeof_addr_;                      // base, free-space, EOF, driver
        // root group symbol table entry
        const uint64_t ste = p;
        root_addr_ = rd(ste + sizeof_addr_, sizeof_addr_);
    } else if (version == 2 || version == 3) {
        sizeof_addr_ = buf_[sb + 9];
        sizeof_len_ = buf_[sb + 10];
        uint64_t p = sb + 12;
        base_ = rd(p, sizeof_addr_);
        p += 3 * sizeof_addr_;                      // base, extension, EOF
        root_addr_ = rd(p, sizeof_addr_);
    } else {
        fail(filename_, "unsupported superblock version " + std::to_string(version));
    }
    if (sizeof_addr_ != 4 && sizeof_addr_ != 8) fail(filename_, "unsupported address size");
    if (sizeof_len_ != 4 && sizeof_len_ != 8) fail(filename_, "unsupported length size");
    (void)object(root_addr_);
}

void File::need(uint64_t off, uint64_t n) const {
    if (off > buf_.size() || n > buf_.size() - off) fail(filename_, "truncated or corrupt file");
}

uint64_t File::rd(uint64_t off, int nbytes) const {
    need(off, nbytes);
    uint64_t v = 0;
    for (int i = 0; i < nbytes; ++i) v |= uint64_t(buf_[off + i]) << (8 * i);
    return v;
}

Datatype File::parse_datatype(uint64_t off, uint64_t* used) const {
    need(off, 8);
    Datatype t;
    const uint8_t b0 = buf_[off];
    t.cls = b0 & 0x0F;
    const int version = b0 >> 4;
    const uint32_t bits = uint32_t(buf_[off + 1]) | (uint32_t(buf_[off + 2]) << 8) | (uint32_t(buf_[off + 3]) << 16);
    t.size = uint32_t(rd(off + 4, 4));
    uint64_t p = off + 8;
    switch (t.cls) {
    case 0:   // fixed point
        t.big_endian = bits & 1;
        t.is_signed = (bits >> 3) & 1;
        p += 4;
        break;
    case 1:   // floating point
        t.big_endian = bits & 1;
        p += 12;
        break;
    case 2:   // time
        p += 2;
        break;
    case 3:   // fixed string
    case 7:   // reference
        break;
    case 4:   // bitfield
        p += 4;
        break;
    case 5: { // opaque: NUL-terminated tag padded to 8
        const uint64_t taglen = bits & 0xFF;
        p += taglen;
        break;
    }
    case 6: { // compound
        const uint32_t n = bits & 0xFFFF;
        for (uint32_t m = 0; m < n; ++m) {
            Datatype::Member mem;
            need(p, 1);
            const uint64_t name_start = p;
            while (true) {
                need(p, 1);
                if (buf_[p] == 0) break;
                mem.name.push_back(char(buf_[p]));
                ++p;
            }
            ++p;   // NUL
            if (version < 3) {
                const uint64_t nlen = p - name_start;
                p = name_start + ((nlen + 7) / 8) * 8;
                mem.offset = uint32_t(rd(p, 4));
                p += 4;
                if (version == 1) p += 1 + 3 + 4 + 4 + 16;
            } else {
                int k = t.size < 256 ? 1 : t.size < 65536 ? 2 : t.size < (1u << 24) ? 3 : 4;
                mem.offset = uint32_t(rd(p, k));
                p += k;
            }
            uint64_t u = 0;
            mem.type = std::make_shared<Datatype>(parse_datatype(p, &u));
            p += u;
            t.members.push_back(mem);
        }
        break;
    }
    case 9: { // variable length
        t.vlen_string = (bits & 0x0F) == 1;
        uint64_t u = 0;
        t.base = std::make_shared<Datatype>(parse_datatype(p, &u));
        p += u;
        break;
    }
    case 10: { // array
        need(p, 1);
        const int rank = buf_[p];
        p += (version < 3) ? 4 : 1;
        p += 4 * rank;
        if (version < 3) p += 4 * rank;
        uint64_t u = 0;
        t.base = std::make_shared<Datatype>(parse_datatype(p, &u));
        p += u;
        break;
    }
    default:
        fail(filename_, "unsupported datatype class " + std::to_string(t.cls));
    }
    *used = p - off;
    return t;
}

static void parse_dataspace(const std::vector<uint8_t>& b, uint64_t off, int sizeof_len,
                            std::vector<uint64_t>* dims, const std::string& fn) {
    if (off + 4 > b.size()) fail(fn, "bad dataspace");
    const int version = b[off];
    const int rank = b[off + 1];
    uint64_t p;
    if (version == 1) {
        p = off + 8;
    } else if (version == 2) {
        p = off + 4;
    } else {
        fail(fn, "unsupported dataspace version");
    }
    dims->clear();
    for (int i = 0; i < rank; ++i) {
        uint64_t v = 0;
        if (p + sizeof_len > b.size()) fail(fn, "bad dataspace");
        for (int k = 0; k < sizeof_len; ++k) v |= uint64_t(b[p + k]) << (8 * k);
        dims->push_back(v);
        p += sizeof_len;
    }
}

void File::parse_message(Object& o, int type, uint64_t off, uint64_t size) const {
    need(off, size);
    switch (type) {
    case 0x0001:
        parse_dataspace(buf_, off, sizeof_len_, &o.dims, filename_);
        o.is_dataset = true;
        break;
    case 0x0003: {
        uint64_t u = 0;
        o.type = parse_datatype(off, &u);
        break;
    }
    case 0x0008: {
        const int version = buf_[off];
        if (version < 3) fail(filename_, "unsupported data layout version");
        o.layout_class = buf_[off + 1];
        if (o.layout_class == 0) {
            const uint64_t n = rd(off + 2, 2);
            need(off + 4, n);
            o.compact.assign(buf_.begin() + off + 4, buf_.begin() + off + 4 + n);
        } else if (o.layout_class == 1) {
            o.data_addr = rd(off + 2, sizeof_addr_);
            o.data_size = rd(off + 2 + sizeof_addr_, sizeof_len_);
        }
        break;
    }
    case 0x000C: {
        Attribute a;
        const int version = buf_[off];
        uint64_t p = off;
        uint64_t nlen, dtlen, dslen;
        if (version == 1 || version == 2) {
            nlen = rd(off + 2, 2);
            dtlen = rd(off + 4, 2);
            dslen = rd(off + 6, 2);
            p = off + 8;
        } else if (version == 3) {
            nlen = rd(off + 2, 2);
            dtlen = rd(off + 4, 2);
            dslen = rd(off + 6, 2);
            p = off + 9;
        } else {
            fail(filename_, "unsupported attribute message version");
        }
        auto pad = [&](uint64_t n) { return version == 1 ? ((n + 7) / 8) * 8 : n; };
        need(p, nlen);
        a.name.assign(reinterpret_cast<const char*>(buf_.data() + p), strnlen(reinterpret_cast<const char*>(buf_.data() + p), nlen));
        p += pad(nlen);
        uint64_t u = 0;
        a.type = parse_datatype(p, &u);
        p += pad(dtlen);
        parse_dataspace(buf_, p, sizeof_len_, &a.dims, filename_);
        p += pad(dslen);
        uint64_t nelem = 1;
        for (auto d : a.dims) nelem *= d;
        const uint64_t nbytes = nelem * a.type.size;
        need(p, nbytes);
        a.data.assign(buf_.begin() + p, buf_.begin() + p + nbytes);
        o.attrs.push_back(std::move(a));
        break;
    }
    case 0x0011:
        o.is_group = true;
        o.has_symtab = true;
        o.btree = rd(off, sizeof_addr_);
        o.heap = rd(off + sizeof_addr_, sizeof_addr_);
        break;
    case 0x0002:
        o.is_group = true;
        break;
    case 0x0006: {   // link message (compact new-style group)
        o.is_group = true;
        const int flags = buf_[off + 1];
        uint64_t p = off + 2;
        int link_type = 0;
        if (flags & 0x08) link_type = buf_[p++];
        if (flags & 0x04) p += 8;
        if (flags & 0x10) p += 1;
        const int lsize = 1 << (flags & 3);
        const uint64_t nlen = rd(p, lsize);
        p += lsize;
        need(p, nlen);
        std::string name(reinterpret_cast<const char*>(buf_.data() + p), nlen);
        p += nlen;
        if (link_type == 0) o.links.emplace_back(name, rd(p, sizeof_addr_));
        break;
    }
    default:
        break;
    }
}

std::shared_ptr<Object> File::object(uint64_t addr) const {
    auto it = cache_.find(addr);
    if (it != cache_.end()) return it->second;
    auto o = std::make_shared<Object>();
    o->addr = addr;
    const uint64_t a = base_ + addr;
    need(a, 16);
    struct Block { uint64_t off, len; };
    std::vector<Block> blocks;
    if (std::memcmp(buf_.data() + a, "OHDR", 4) == 0) {
        const int flags = buf_[a + 5];
        uint64_t p = a + 6;
        if (flags & 0x20) p += 16;
        if (flags & 0x10) p += 4;
        const int csize = 1 << (flags & 3);
        const uint64_t len0 = rd(p, csize);
        p += csize;
        const bool track_order = flags & 0x04;
        std::vector<Block> todo{{p, len0}};
        while (!todo.empty()) {
            Block blk = todo.back();
            todo.pop_back();
            uint64_t q = blk.off;
            const uint64_t end = blk.off + blk.len;
            while (q + 4 <= end) {
                const int type = buf_[q];
                const uint64_t size = rd(q + 1, 2);
                q += 4 + (track_order ? 2 : 0);
                if (q + size > end) break;
                if (type == 0x10) {
                    const uint64_t caddr = rd(q, sizeof_addr_);
                    const uint64_t clen = rd(q + sizeof_addr_, sizeof_len_);
                    // OCHK signature (4) ... checksum (4)
                    todo.push_back({base_ + caddr + 4, clen - 8});
                } else {
                    parse_message(*o, type, q, size);
                }
                q += size;
            }
        }
    } else {
        const int version = buf_[a];
        if (version != 1) fail(filename_, "unsupported object header version");
        const uint64_t nmsgs = rd(a + 2, 2);
        const uint64_t hsize = rd(a + 8, 4);
        std::vector<Block> todo{{a + 16, hsize}};
        uint64_t seen = 0;
        while (!todo.empty() && seen < nmsgs) {
            Block blk = todo.front();
            todo.erase(todo.begin());
            uint64_t q = blk.off;
            const uint64_t end = blk.off + blk.len;
            while (q + 8 <= end && seen < nmsgs) {
                const int type = int(rd(q, 2));
                const uint64_t size = rd(q + 2, 2);
                q += 8;
                if (q + size > end) fail(filename_, "corrupt object header");
                ++seen;
                if (type == 0x10) {
                    todo.push_back({base_ + rd(q, sizeof_addr_), rd(q + sizeof_addr_, sizeof_len_)});
                } else {
                    parse_message(*o, type, q, size);
                }
                q += size;
            }
        }
    }
    if (o->is_group) o->is_dataset = false;
    cache_[addr] = o;
    return o;
}

std::string File::heap_name(uint64_t heap_addr, uint64_t offset) const {
    const uint64_t h = base_ + heap_addr;
    need(h, 8);
    if (std::memcmp(buf_.data() + h, "HEAP", 4) != 0) fail(filename_, "bad local heap");
    const uint64_t data_size = rd(h + 8, sizeof_len_);
    const uint64_t data_addr = rd(h + 8 + 2 * sizeof_len_, sizeof_addr_);
    if (offset >= data_size) fail(filename_, "bad local heap offset");
    const uint64_t p = base_ + data_addr + offset;
    need(p, data_size - offset);
    return std::string(reinterpret_cast<const char*>(buf_.data() + p), strnlen(reinterpret_cast<const char*>(buf_.data() + p), data_size - offset));
}

uint64_t File::lookup_child(const Object& g, const std::string& name) const {
    for (auto& l : g.links)
        if (l.first == name) return l.second;
    if (!g.has_symtab) return 0;
    // Depth-first walk over the group's v1 B-tree; leaves point at SNODs.
    std::vector<uint64_t> nodes{g.btree};
    int guard = 0;
    while (!nodes.empty()) {
        if (++guard > 100000) fail(filename_, "B-tree walk did not terminate");
        const uint64_t n = base_ + nodes.back();
        nodes.pop_back();
        need(n, 8);
        if (std::memcmp(buf_.data() + n, "TREE", 4) != 0) fail(filename_, "bad B-tree node");
        const int level = buf_[n + 5];
        const uint64_t used = rd(n + 6, 2);
        uint64_t p = n + 8 + 2 * sizeof_addr_ + sizeof_len_;   // first child
        for (uint64_t i = 0; i < used; ++i) {
            const uint64_t child = rd(p, sizeof_addr_);
            p += sizeof_addr_ + sizeof_len_;
            if (level > 0) {
                nodes.push_back(child);
                continue;
            }
            const uint64_t s = base_ + child;
            need(s, 8);
            if (std::memcmp(buf_.data() + s, "SNOD", 4) != 0) fail(filename_, "bad symbol table node");
            const uint64_t nsym = rd(s + 6, 2);
            const uint64_t esize = 2 * sizeof_addr_ + 8 + 16;
            for (uint64_t e = 0; e < nsym; ++e) {
                const uint64_t ep = s + 8 + e * esize;
                if (heap_name(g.heap, rd(ep, sizeof_addr_)) == name) return rd(ep + sizeof_addr_, sizeof_addr_);
            }
        }
    }
    return 0;
}

uint64_t File::resolve(const std::string& path) const {
    uint64_t addr = root_addr_;
    for (const auto& part : split_path(path)) {
        auto o = object(addr);
        if (!o->is_group) return 0;
        addr = lookup_child(*o, part);
        if (addr == 0) return 0;
    }
    return addr;
}

bool File::exists(const std::string& path) const {
    try {
        return resolve(path) != 0;
    } catch (const std::exception&) {
        return false;
    }
}

std::vector<uint8_t> File::global_heap_object(uint64_t collection, uint32_t index) const {
    const uint64_t c = base_ + collection;
    need(c, 16);
    if (std::memcmp(buf_.data() + c, "GCOL", 4) != 0) fail(filename_, "bad global heap collection");
    const uint64_t csize = rd(c + 8, sizeof_len_);
    need(c, csize);
    uint64_t p = c + 8 + sizeof_len_;
    while (p + 8 + sizeof_len_ <= c + csize) {
        const uint32_t idx = uint32_t(rd(p, 2));
        const uint64_t size = rd(p + 8, sizeof_len_);
        const uint64_t data = p + 8 + sizeof_len_;
        if (idx == 0) break;
        if (idx == index) {
            need(data, size);
            return std::vector<uint8_t>(buf_.begin() + data, buf_.begin() + data + size);
        }
        p = data + ((size + 7) / 8) * 8;
    }
    fail(filename_, "global heap object not found");
}

std::string File::decode_string(const Datatype& t, const uint8_t* p) const {
    if (t.cls == 3) {
        std::string s(reinterpret_cast<const char*>(p), strnlen(reinterpret_cast<const char*>(p), t.size));
        while (!s.empty() && s.back() == ' ') s.pop_back();
        return s;
    }
    if (t.cls == 9) {
        uint32_t len = 0;
        std::memcpy(&len, p, 4);
        uint64_t coll = 0;
        for (int i = 0; i < sizeof_addr_; ++i) coll |= uint64_t(p[4 + i]) << (8 * i);
        uint32_t idx = 0;
        std::memcpy(&idx, p + 4 + sizeof_addr_, 4);
        if (coll == 0 && len == 0) return std::string();
        auto bytes = global_heap_object(coll, idx);
        const size_t n = std::min<size_t>(len, bytes.size());
        std::string s(reinterpret_cast<const char*>(bytes.data()), n);
        const size_t z = s.find('\0');
        if (z != std::string::npos) s.resize(z);
        return s;
    }
    fail(filename_, "attribute is not a string");
}

double File::decode_number(const Datatype& t, const uint8_t* p) const {
    uint8_t tmp[8];
    if (t.size > 8) fail(filename_, "number too wide");
    for (uint32_t i = 0; i < t.size; ++i) tmp[i] = t.big_endian ? p[t.size - 1 - i] : p[i];
    if (t.cls == 1) {
        if (t.size == 4) {
            float f;
            std::memcpy(&f, tmp, 4);
            return f;
        }
        if (t.size == 8) {
            double d;
            std::memcpy(&d, tmp, 8);
            return d;
        }
    } else if (t.cls == 0) {
        uint64_t v = 0;
        for (uint32_t i = 0; i < t.size; ++i) v |= uint64_t(tmp[i]) << (8 * i);
        if (t.is_signed && t.size < 8 && (v >> (8 * t.size - 1)) & 1) v |= ~uint64_t(0) << (8 * t.size);
        return t.is_signed ? double(int64_t(v)) : double(v);
    }
    fail(filename_, "unsupported numeric type");
}

const Attribute* File::find_attribute(const std::string& path, const std::string& name) const {
    const uint64_t addr = resolve(path);
    if (addr == 0) return nullptr;
    auto o = object(addr);
    for (auto& a : o->attrs)
        if (a.name == name) return &a;
    return nullptr;
}

bool File::has_attribute(const std::string& path, const std::string& name) const {
    return find_attribute(path, name) != nullptr;
}

std::string File::attribute_string(const std::string& path, const std::string& name) const {
    const Attribute* a = find_attribute(path, name);
    if (!a) fail(filename_, "no attribute '" + name + "' on '" + path + "'");
    if (a->data.size() < a->type.size) fail(filename_, "empty attribute '" + name + "'");
    return decode_string(a->type, a->data.data());
}

void File::attribute_quantity(const std::string& path, const std::string& name, double* value,
                              std::string* unit) const {
    const Attribute* a = find_attribute(path, name);
    if (!a) fail(filename_, "no attribute '" + name + "' on '" + path + "'");
    if (a->type.cls != 6) fail(filename_, "attribute '" + name + "' is not a {value, unit} compound");
    const Datatype::Member* mv = nullptr;
    const Datatype::Member* mu = nullptr;
    for (auto& m : a->type.members) {
        if (m.name == "value") mv = &m;
        if (m.name == "unit") mu = &m;
    }
    if (!mv || !mu) fail(filename_, "attribute '" + name + "' lacks value/unit members");
    *value = decode_number(*mv->type, a->data.data() + mv->offset);
    *unit = decode_string(*mu->type, a->data.data() + mu->offset);
}

std::vector<double> File::read_dataset(const std::string& path, std::vector<uint64_t>* dims) const {
    const uint64_t addr = resolve(path);
    if (addr == 0) fail(filename_, "no dataset '" + path + "'");
    auto o = object(addr);
    if (!o->is_dataset) fail(filename_, "'" + path + "' is not a dataset");
    uint64_t n = 1;
    for (auto d : o->dims) n *= d;
    const uint8_t* src;
    if (o->layout_class == 1) {
        if (o->data_addr == UINT64_MAX || (n > 0 && o->data_addr == 0 && o->data_size == 0)) {
            fail(filename_, "dataset '" + path + "' has no storage");
        }
        need(base_ + o->data_addr, n * o->type.size);
        src = buf_.data() + base_ + o->data_addr;
    } else if (o->layout_class == 0) {
        if (o->compact.size() < n * o->type.size) fail(filename_, "short compact dataset");
        src = o->compact.data();
    } else {
        fail(filename_, "dataset '" + path + "': only contiguous/compact storage is supported");
    }
    std::vector<double> out(n);
    for (uint64_t i = 0; i < n; ++i) out[i] = decode_number(o->type, src + i * o->type.size);
    if (dims) *dims = o->dims;
    return out;
}

bool File::dimension_scale(const std::string& path, int dim, std::vector<double>* values,
                           std::string* units) const {
    const Attribute* a = find_attribute(path, "DIMENSION_LIST");
    if (!a) return false;
    if (a->type.cls != 9 || a->dims.empty() || uint64_t(dim) >= a->dims[0]) return false;
    const uint8_t* p = a->data.data() + size_t(dim) * a->type.size;
    uint32_t len = 0;
    std::memcpy(&len, p, 4);
    if (len == 0) return false;
    uint64_t coll = 0;
    for (int i = 0; i < sizeof_addr_; ++i) coll |= uint64_t(p[4 + i]) << (8 * i);
    uint32_t idx = 0;
    std::memcpy(&idx, p + 4 + sizeof_addr_, 4);
    auto refs = global_heap_object(coll, idx);
    if (refs.size() < size_t(sizeof_addr_)) fail(filename_, "bad DIMENSION_LIST reference");
    uint64_t target = 0;
    for (int i = 0; i < sizeof_addr_; ++i) target |= uint64_t(refs[i]) << (8 * i);
    auto s = object(target);
    if (!s->is_dataset) fail(filename_, "dimension scale is not a dataset");
    // read through a temporary path-less accessor
    uint64_t n = 1;
    for (auto d : s->dims) n *= d;
    const uint8_t* src;
    if (s->layout_class == 1) {
        need(base_ + s->data_addr, n * s->type.size);
        src = buf_.data() + base_ + s->data_addr;
    } else if (s->layout_class == 0) {
        src = s->compact.data();
    } else {
        fail(filename_, "dimension scale storage not supported");
    }
    values->resize(n);
    for (uint64_t i = 0; i < n; ++i) (*values)[i] = decode_number(s->type, src + i * s->type.size);
    units->clear();
    for (auto& at : s->attrs)
        if (at.name == "units") *units = decode_string(at.type, at.data.data());
    return true;
}

}  // namespace h5
}  // namespace nbx
