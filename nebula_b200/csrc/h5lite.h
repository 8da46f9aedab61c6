// Read-only access to the subset of HDF5 that Nebula material (.mat) files use.
//
// Nebula's material loader (source/io/hdf5_file.{h,cpp}) reads root
// attributes (variable-length strings, and compound {double value; vlen
// string unit} quantities), float/double datasets with a "units" attribute,
// and the axis of each dimension through the HDF5 dimension-scale
// DIMENSION_LIST attribute.  This reader implements those structures from the
// HDF5 File Format Specification without libhdf5:
//   * superblock versions 0, 1, 2 and 3;
//   * object headers version 1 (with continuation blocks) and version 2
//     ("OHDR"/"OCHK");
//   * groups stored as a symbol table (v1 B-tree + SNOD + local heap) or as
//     compact link messages;
//   * contiguous and compact dataset layouts (chunked storage is rejected with
//     an error);
//   * fixed-point, floating-point, fixed and variable-length string,
//     compound, object-reference and variable-length-sequence datatypes;
//   * global heap collections for variable-length data.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace nbx {
namespace h5 {

struct Datatype {
    int cls = -1;          // HDF5 datatype class
    uint32_t size = 0;     // element size in the file
    bool is_signed = false;
    bool big_endian = false;
    bool vlen_string = false;
    std::shared_ptr<Datatype> base;   // vlen / array base type
    struct Member {
        std::string name;
        uint32_t offset;
        std::shared_ptr<Datatype> type;
    };
    std::vector<Member> members;      // compound members
};

struct Attribute {
    std::string name;
    Datatype type;
    std::vector<uint64_t> dims;       // empty: scalar
    std::vector<uint8_t> data;        // raw file bytes
};

struct Object {
    uint64_t addr = 0;
    bool is_group = false;
    bool is_dataset = false;
    // group
    uint64_t btree = 0, heap = 0;
    bool has_symtab = false;
    std::vector<std::pair<std::string, uint64_t>> links;   // compact links
    // dataset
    Datatype type;
    std::vector<uint64_t> dims;
    int layout_class = -1;
    uint64_t data_addr = 0, data_size = 0;
    std::vector<uint8_t> compact;
    std::vector<Attribute> attrs;
};

class File {
public:
    explicit File(const std::string& filename);   // throws std::runtime_error

    const std::string& filename() const { return filename_; }

    // True if `path` names a group or dataset ("/a/b", "a/b").
    bool exists(const std::string& path) const;

    // Attribute of the object at `path` ("/" is the root group).
    bool has_attribute(const std::string& path, const std::string& name) const;
    std::string attribute_string(const std::string& path, const std::string& name) const;
    // Compound {double value; string unit} attribute.
    void attribute_quantity(const std::string& path, const std::string& name,
                            double* value, std::string* unit) const;

    // Dataset contents converted to double, row-major; dims returned.
    std::vector<double> read_dataset(const std::string& path, std::vector<uint64_t>* dims) const;

    // First dimension scale attached to dimension `dim` of the dataset.
    // Returns false if the dataset has no scale attached to that dimension.
    bool dimension_scale(const std::string& path, int dim, std::vector<double>* values,
                         std::string* units) const;

private:
    std::string filename_;
    std::vector<uint8_t> buf_;
    int sizeof_addr_ = 8, sizeof_len_ = 8;
    uint64_t base_ = 0;
    uint64_t root_addr_ = 0;
    mutable std::map<uint64_t, std::shared_ptr<Object>> cache_;

    uint64_t rd(uint64_t off, int nbytes) const;
    void need(uint64_t off, uint64_t n) const;
    std::shared_ptr<Object> object(uint64_t addr) const;
    void parse_message(Object& o, int type, uint64_t off, uint64_t size) const;
    Datatype parse_datatype(uint64_t off, uint64_t* used) const;
    uint64_t lookup_child(const Object& group, const std::string& name) const;
    uint64_t resolve(const std::string& path) const;   // 0 if missing
    std::string heap_name(uint64_t heap_addr, uint64_t offset) const;
    std::vector<uint8_t> global_heap_object(uint64_t collection, uint32_t index) const;
    const Attribute* find_attribute(const std::string& path, const std::string& name) const;
    std::string decode_string(const Datatype& t, const uint8_t* p) const;
    double decode_number(const Datatype& t, const uint8_t* p) const;
};

}  // namespace h5
}  // namespace nbx
