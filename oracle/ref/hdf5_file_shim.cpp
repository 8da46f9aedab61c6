// Test infrastructure: implementation of the reference's nbl::hdf5_file API
// (declared in source/io/hdf5_file.h) for building the reference CPU path in
// an environment without libhdf5.  Only source/io/hdf5_file.cpp is replaced;
// every other reference file is compiled unmodified from its own location.
//
// Reading is delegated to nebula_b200/csrc/h5lite; the semantics follow
// source/io/hdf5_file.cpp: attributes on the root group, "units" attributes
// parsed with the caller's unit_parser, dimension scales checked for linear /
// logarithmic spacing and returned as util::linspace / util::geomspace.
#include "config/config.h"
#include "io/hdf5_file.h"

#include <map>
#include <memory>
#include <mutex>

#include "h5lite.h"

namespace nbl {

namespace {
std::mutex g_mutex;
std::map<hid_t, std::unique_ptr<nbx::h5::File>> g_files;
hid_t g_next = 1;

nbx::h5::File& file_of(hid_t id) {
    std::lock_guard<std::mutex> lk(g_mutex);
    return *g_files.at(id);
}

std::pair<std::vector<double>, units::quantity<double>> scale_of(
    nbx::h5::File& f, std::string const& dataset, int dim, units::unit_parser<double> const& parser) {
    std::vector<double> values;
    std::string unit;
    if (!f.dimension_scale(dataset, dim, &values, &unit)) return {values, units::quantity<double>()};
    return {values, parser.parse_unit(unit)};
}

template<typename T, typename table_t>
void fill(nbx::h5::File& f, std::string const& name, table_t& table, size_t n) {
    std::vector<uint64_t> dims;
    auto v = f.read_dataset(name, &dims);
    if (v.size() != n) throw std::runtime_error("Could not read table '" + name + '\'');
    T* dst = table.data();
    for (size_t i = 0; i < n; ++i) dst[i] = T(v[i]);
}

std::vector<uint64_t> dims_of(nbx::h5::File& f, std::string const& name, size_t rank) {
    std::vector<uint64_t> dims;
    if (!f.exists(name)) throw std::runtime_error("Could not read table '" + name + '\'');
    f.read_dataset(name, &dims);
    if (dims.size() != rank) throw std::runtime_error("Dataspace has unexpected dimension");
    return dims;
}
}  // namespace

hdf5_file::hdf5_file(std::string const& filename) : _filename(filename) {
    std::unique_ptr<nbx::h5::File> f;
    try {
        f.reset(new nbx::h5::File(filename));
    } catch (std::exception const&) {
        throw std::runtime_error("Unable to open file " + filename);
    }
    std::lock_guard<std::mutex> lk(g_mutex);
    _file = g_next++;
    g_files[_file] = std::move(f);
}

hdf5_file::~hdf5_file() {
    std::lock_guard<std::mutex> lk(g_mutex);
    g_files.erase(_file);
}

std::string const& hdf5_file::get_filename() const { return _filename; }

bool hdf5_file::exists(std::string const& name) const { return file_of(_file).exists(name); }

std::string hdf5_file::get_property_string(std::string const& name) const {
    auto& f = file_of(_file);
    if (!f.has_attribute("/", name)) throw std::runtime_error("Could not read string property '" + name + '\'');
    return f.attribute_string("/", name);
}

units::quantity<double> hdf5_file::get_property_quantity(std::string const& name,
                                                         units::unit_parser<double> const& parser) const {
    auto& f = file_of(_file);
    if (!f.has_attribute("/", name)) throw std::runtime_error("Could not read quantity property '" + name + '\'');
    double value;
    std::string unit;
    f.attribute_quantity("/", name, &value, &unit);
    return value * parser.parse_unit(unit);
}

std::string hdf5_file::get_property_string(std::string const& name, std::string const& _default) const {
    auto& f = file_of(_file);
    if (!f.has_attribute("/", name)) return _default;
    return f.attribute_string("/", name);
}

units::quantity<double> hdf5_file::get_property_quantity(std::string const& name,
                                                         units::quantity<double> const& _default,
                                                         units::unit_parser<double> const& parser) const {
    auto& f = file_of(_file);
    if (!f.has_attribute("/", name)) return _default;
    double value;
    std::string unit;
    f.attribute_quantity("/", name, &value, &unit);
    return value * parser.parse_unit(unit);
}

template<typename T>
util::table_1D<T, false> hdf5_file::fill_table1D(std::string const& dataset_name) const {
    auto& f = file_of(_file);
    auto d = dims_of(f, dataset_name, 1);
    auto table = util::table_1D<T, false>::create(0, 1, int(d[0]));
    fill<T>(f, dataset_name, table, d[0]);
    return table;
}

template<typename T>
util::table_2D<T, false> hdf5_file::fill_table2D(std::string const& dataset_name) const {
    auto& f = file_of(_file);
    auto d = dims_of(f, dataset_name, 2);
    auto table = util::table_2D<T, false>::create(0, 1, int(d[0]), 0, 1, int(d[1]));
    fill<T>(f, dataset_name, table, d[0] * d[1]);
    return table;
}

template<typename T>
util::table_3D<T, false> hdf5_file::fill_table3D(std::string const& dataset_name) const {
    auto& f = file_of(_file);
    auto d = dims_of(f, dataset_name, 3);
    auto table = util::table_3D<T, false>::create(0, 1, int(d[0]), 0, 1, int(d[1]), 0, 1, int(d[2]));
    fill<T>(f, dataset_name, table, d[0] * d[1] * d[2]);
    return table;
}

util::linspace<units::quantity<double>> hdf5_file::get_lin_dimscale(std::string const& dataset_name, int dim,
                                                                   int N_expected,
                                                                   units::unit_parser<double> const& parser) const {
    auto& f = file_of(_file);
    if (!f.exists(dataset_name)) throw std::runtime_error("Could not read table '" + dataset_name + '\'');
    auto s = scale_of(f, dataset_name, dim, parser);
    if (s.first.size() == 0)
        return util::linspace<units::quantity<double>>(0 * units::dimensionless, 1 * units::dimensionless, N_expected);
    if (s.first.size() != (size_t)N_expected) throw std::runtime_error("Dimension scale has unexpected size.");
    util::linspace<double> check(s.first.front(), s.first.back(), N_expected);
    for (int i = 0; i < N_expected; ++i)
        if (check[i] - s.first[i] > EPSILON)
            throw std::runtime_error("Dataset " + dataset_name + ": Linear dimension scale expected");
    return util::linspace<units::quantity<double>>(s.first.front() * s.second, s.first.back() * s.second, N_expected);
}

util::geomspace<units::quantity<double>> hdf5_file::get_log_dimscale(std::string const& dataset_name, int dim,
                                                                    int N_expected,
                                                                    units::unit_parser<double> const& parser) const {
    auto& f = file_of(_file);
    if (!f.exists(dataset_name)) throw std::runtime_error("Could not read table '" + dataset_name + '\'');
    auto s = scale_of(f, dataset_name, dim, parser);
    if (s.first.size() != (size_t)N_expected) throw std::runtime_error("Dimension scale has unexpected size.");
    util::geomspace<double> check(s.first.front(), s.first.back(), N_expected);
    for (int i = 0; i < N_expected; ++i)
        if (check[i] - s.first[i] > EPSILON)
            throw std::runtime_error("Dataset " + dataset_name + ": Logarithmic dimension scale expected");
    return util::geomspace<units::quantity<double>>(s.first.front() * s.second, s.first.back() * s.second, N_expected);
}

units::quantity<double> hdf5_file::get_unit(std::string const& dataset_name,
                                            units::unit_parser<double> const& parser) const {
    auto& f = file_of(_file);
    if (!f.exists(dataset_name)) throw std::runtime_error("Could not read table '" + dataset_name + '\'');
    return parser.parse_unit(f.attribute_string(dataset_name, "units"));
}

template util::table_1D<float, false> hdf5_file::fill_table1D(std::string const&) const;
template util::table_2D<float, false> hdf5_file::fill_table2D(std::string const&) const;
template util::table_3D<float, false> hdf5_file::fill_table3D(std::string const&) const;
template util::table_1D<double, false> hdf5_file::fill_table1D(std::string const&) const;
template util::table_2D<double, false> hdf5_file::fill_table2D(std::string const&) const;
template util::table_3D<double, false> hdf5_file::fill_table3D(std::string const&) const;

}  // namespace nbl
