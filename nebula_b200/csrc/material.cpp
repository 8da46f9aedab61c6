// Kieft & Bosch material loader; see material.h for the reference lines followed.
#include "material.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <map>
#include <stdexcept>

#include "h5lite.h"

namespace nbx {

namespace {
constexpr float kEpsilon = 10 * std::numeric_limits<float>::epsilon();

Quantity make_q(double v, int e, int l, int t, int T, int c) {
    Quantity q;
    q.value = v;
    q.dim[0] = e;
    q.dim[1] = l;
    q.dim[2] = t;
    q.dim[3] = T;
    q.dim[4] = c;
    return q;
}

const std::map<std::string, Quantity>& unit_table() {
    // Values of source/common/units/unit_system.h: eV, nm and ns are the base
    // units; mass is energy * time^2 / length^2.
    static const std::map<std::string, Quantity> t = {
        {"eV", make_q(1, 1, 0, 0, 0, 0)},
        {"nm", make_q(1, 0, 1, 0, 0, 0)},
        {"K", make_q(1, 0, 0, 0, 1, 0)},
        {"s", make_q(1e9, 0, 0, 1, 0, 0)},
        {"m", make_q(1e9, 0, 1, 0, 0, 0)},
        {"cm", make_q(1e7, 0, 1, 0, 0, 0)},
        {"g", make_q(6.2415e15, 1, -2, 2, 0, 0)},
        {"C", make_q(6.2415e18, 0, 0, 0, 0, 1)},
        {"radian", make_q(1, 0, 0, 0, 0, 0)},
    };
    return t;
}

bool same_dim(const Quantity& a, const Quantity& b) {
    for (int i = 0; i < 5; ++i)
        if (a.dim[i] != b.dim[i]) return false;
    return true;
}

double as_double(const Quantity& q, const std::string& what) {
    if (!q.dimensionless()) throw std::runtime_error("Can only convert dimensionless quantity (" + what + ")");
    return q.value;
}

const Quantity kEV = make_q(1, 1, 0, 0, 0, 0);
const Quantity kNM = make_q(1, 0, 1, 0, 0, 0);

Quantity mul(const Quantity& a, const Quantity& b) {
    Quantity r = a;
    r.value = a.value * b.value;
    for (int i = 0; i < 5; ++i) r.dim[i] = a.dim[i] + b.dim[i];
    return r;
}
Quantity div(const Quantity& a, const Quantity& b) {
    Quantity r = a;
    r.value = a.value / b.value;
    for (int i = 0; i < 5; ++i) r.dim[i] = a.dim[i] - b.dim[i];
    return r;
}

// hdf5_file::get_property_quantity: value * parse(unit)
Quantity property(const h5::File& f, const std::string& name) {
    double v;
    std::string u;
    f.attribute_quantity("/", name, &v, &u);
    Quantity q = parse_unit(u);
    q.value = q.value * v;
    return q;
}

Quantity dataset_unit(const h5::File& f, const std::string& path) {
    return parse_unit(f.attribute_string(path, "units"));
}

// geomspace / linspace of quantities as hdf5_file::get_{log,lin}_dimscale
// return them (source/io/hdf5_file.cpp:291-359, source/common/util/range.h).
struct Axis {
    double first = 0, step = 0;
    bool log = false;
    size_t n = 0;
    Quantity dim;   // the scale's unit dimension (value 1)
    double at(size_t i) const { return log ? first * std::exp(i * step) : first + i * step; }
    double front() const { return first; }
    double back() const { return at(n - 1); }
    Quantity unit_front() const { Quantity q = dim; q.value = front(); return q; }
    Quantity unit_back() const { Quantity q = dim; q.value = back(); return q; }
};

Axis dimscale(const h5::File& f, const std::string& path, int dim, int n_expected, bool logarithmic) {
    std::vector<double> values;
    std::string units;
    const bool found = f.dimension_scale(path, dim, &values, &units);
    Axis a;
    a.n = size_t(n_expected);
    a.log = logarithmic;
    if (!found || values.empty()) {
        if (logarithmic) throw std::runtime_error("Dimension scale has unexpected size.");
        a.first = 0;
        a.step = (1.0 - 0.0) / (n_expected - 1);
        return a;
    }
    if (values.size() != size_t(n_expected)) throw std::runtime_error("Dimension scale has unexpected size.");
    const Quantity u = parse_unit(units);
    a.dim = u;
    a.dim.value = 1;
    // Spacing check on the raw values (one-sided, as the reference does).
    Axis chk;
    chk.n = values.size();
    chk.log = logarithmic;
    chk.first = values.front();
    chk.step = logarithmic ? std::log(values.back() / values.front()) / (n_expected - 1)
                           : (values.back() - values.front()) / (n_expected - 1);
    for (int i = 0; i < n_expected; ++i)
        if (chk.at(size_t(i)) - values[size_t(i)] > kEpsilon)
            throw std::runtime_error("Dataset " + path + (logarithmic ? ": Logarithmic" : ": Linear") +
                                     " dimension scale expected");
    const double start = u.value * values.front();
    const double stop = u.value * values.back();
    a.first = start;
    a.step = logarithmic ? std::log(stop / start) / (n_expected - 1) : (stop - start) / (n_expected - 1);
    return a;
}

Table1D read_table1d(const h5::File& f, const std::string& path) {
    std::vector<uint64_t> dims;
    auto v = f.read_dataset(path, &dims);
    if (dims.size() != 1) throw std::runtime_error("Dataspace has unexpected dimension");
    Table1D t;
    t.n = int(dims[0]);
    t.data.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) t.data[i] = float(v[i]);
    t.x_min = 0;
    t.x_step = float(t.n - 1) / (1.0f - 0.0f);
    return t;
}

Table2D read_table2d(const h5::File& f, const std::string& path) {
    std::vector<uint64_t> dims;
    auto v = f.read_dataset(path, &dims);
    if (dims.size() != 2) throw std::runtime_error("Dataspace has unexpected dimension");
    Table2D t;
    t.width = int(dims[0]);
    t.height = int(dims[1]);
    t.data.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) t.data[i] = float(v[i]);
    return t;
}

Table3D read_table3d(const h5::File& f, const std::string& path) {
    std::vector<uint64_t> dims;
    auto v = f.read_dataset(path, &dims);
    if (dims.size() != 3) throw std::runtime_error("Dataspace has unexpected dimension");
    Table3D t;
    t.width = int(dims[0]);
    t.height = int(dims[1]);
    t.depth = int(dims[2]);
    t.data.resize(v.size());
    for (size_t i = 0; i < v.size(); ++i) t.data[i] = float(v[i]);
    return t;
}

// table_3D::set_scale (source/common/util/table_3D.inl:155-166)
void set_scale(Table3D& t, float x_min, float x_max, float y_min, float y_max, float z_min, float z_max) {
    t.x_min = x_min;
    t.x_step = (t.width - 1) / (x_max - x_min);
    t.y_min = y_min;
    t.y_step = (t.height - 1) / (y_max - y_min);
    t.z_min = z_min;
    t.z_step = (t.depth - 1) / (z_max - z_min);
}

// units::quantity -> scalar conversion (source/common/units/quantity.h:32-37)
double scalar(const Quantity& q, const std::string& what) {
    if (!q.dimensionless()) throw std::runtime_error("Can only convert dimensionless quantity to scalar (" + what + ")");
    return q.value;
}

void set_scale(Table1D& t, const Axis& x) {
    const float x_min = float(std::log(x.front() / kEV.value));
    const float x_max = float(std::log(x.back() / kEV.value));
    t.x_min = x_min;
    t.x_step = (t.n - 1) / (x_max - x_min);
}

void set_scale(Table2D& t, float x_min, float x_max, float y_min, float y_max) {
    t.x_min = x_min;
    t.x_step = (t.width - 1) / (x_max - x_min);
    t.y_min = y_min;
    t.y_step = (t.height - 1) / (y_max - y_min);
}

void load_log_imfp(const h5::File& f, const std::string& path, Table1D* t) {
    *t = read_table1d(f, path);
    const Axis K = dimscale(f, path, 0, t->n, true);
    set_scale(*t, K);
    const Quantity u = mul(dataset_unit(f, path), kNM);
    const float unit = float(as_double(u, path + " units"));
    for (int x = 0; x < t->n; ++x) t->data[size_t(x)] = std::log(t->data[size_t(x)] * unit);
}

// full_penn::create (source/physics/full_penn.h:296-392), operation for
// operation: float products where the reference multiplies two reals, double
// where it works on quantities.
void load_penn(const h5::File& f, const Quantity& fermi_q, MaterialTables* m) {
    load_log_imfp(f, "/full_penn/imfp", &m->penn_imfp);
    {
        const std::string path = "/full_penn/omega_icdf";
        Table2D& t = m->penn_omega_icdf;
        t = read_table2d(f, path);
        const Axis K = dimscale(f, path, 0, t.width, true);
        const Axis P = dimscale(f, path, 1, t.height, false);
        set_scale(t, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(P.front()), float(P.back()));
        const float unit = float(as_double(div(dataset_unit(f, path), kEV), path + " units"));
        for (int x = 0; x < t.width; ++x) {
            const double K_x = K.at(size_t(x));
            for (int y = 0; y < t.height; ++y) {
                float& v = t.data[size_t(x) * t.height + y];
                const double a = (K_x - fermi_q.value) / kEV.value;
                const double b = double(v * unit);
                v = float(std::log(std::max(0.0, std::min<double>(a, b))));
            }
        }
    }
    {
        const std::string path = "/full_penn/q_icdf";
        Table3D& t = m->penn_q_icdf;
        t = read_table3d(f, path);
        const Axis K = dimscale(f, path, 0, t.width, true);
        const Axis W = dimscale(f, path, 1, t.height, false);
        const Axis P = dimscale(f, path, 2, t.depth, false);
        set_scale(t, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(W.front()), float(W.back()), float(P.front()), float(P.back()));
        // hbar / sqrt(2 m_e) = 0.19519 nm eV^1/2; the product must be dimensionless
        Quantity u = dataset_unit(f, path);
        u.value = u.value * 0.19519;
        const float unit = float(scalar(mul(u, kNM), path + " units"));
        for (auto& v : t.data) v = v * unit;
    }
    {
        const std::string path = "/ionization/binding_icdf";
        Table3D& t = m->penn_ionisation;
        t = read_table3d(f, path);
        const Axis K = dimscale(f, path, 0, t.width, true);
        const Axis O = dimscale(f, path, 1, t.height, true);
        const Axis P = dimscale(f, path, 2, t.depth, false);
        set_scale(t, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(std::log(scalar(O.unit_front(), path + " omega axis"))),
                  float(std::log(scalar(O.unit_back(), path + " omega axis"))), float(P.front()), float(P.back()));
        const float unit = float(as_double(div(dataset_unit(f, path), kEV), path + " units"));
        for (auto& v : t.data) {
            float binding = v * unit;
            if (binding < 50 || !std::isfinite(binding)) binding = -1;
            v = binding;
        }
    }
}
}  // namespace

bool Quantity::dimensionless() const {
    for (int d : dim)
        if (d != 0) return false;
    return true;
}

Quantity parse_unit(const std::string& text) {
    Quantity result;
    size_t pos = 0;
    const auto& table = unit_table();
    auto is_new = [](char c) { return c == '*' || c == '/'; };
    while (pos < text.size()) {
        int power = text[pos] == '/' ? -1 : 1;
        if (is_new(text[pos])) ++pos;
        std::string name;
        while (pos < text.size() && text[pos] != '^' && !is_new(text[pos])) name.push_back(text[pos++]);
        auto it = table.find(name);
        if (it == table.end()) throw std::runtime_error("Unknown unit '" + name + "'.");
        if (pos < text.size() && text[pos] == '^') {
            std::string p;
            for (++pos; pos < text.size() && !is_new(text[pos]); ++pos) p.push_back(text[pos]);
            power *= std::stoi(p);
        }
        Quantity u = it->second;
        u.value = std::pow(u.value, power);
        for (int i = 0; i < 5; ++i) u.dim[i] *= power;
        result = mul(result, u);
    }
    return result;
}

float table2d_get_rounddown(const Table2D& t, float x, float y) {
    const float x_index = (x - t.x_min) * t.x_step;
    const float y_index = (y - t.y_min) * t.y_step;
    int low_x = int(std::floor(x_index));
    int low_y = int(std::floor(y_index));
    low_x = low_x < 0 ? 0 : (low_x > t.width - 1 ? t.width - 1 : low_x);
    low_y = low_y < 0 ? 0 : (low_y > t.height - 1 ? t.height - 1 : low_y);
    return t.at(low_x, low_y);
}

float MaterialTables::max_energy(bool penn) const {
    float e = std::numeric_limits<float>::infinity();
    const float ein = std::exp((penn ? penn_imfp : in_imfp).get_scalemax());
    if (ein < e) e = ein;
    const float eel = std::exp(el_imfp.get_scalemax());
    if (eel < e) e = eel;
    return e;
}

MaterialTables load_material(const std::string& filename) {
    h5::File f(filename);
    MaterialTables m;
    m.filename = filename;
    m.name = f.has_attribute("/", "name") ? f.attribute_string("/", "name") : std::string();
    m.cstool_version = f.has_attribute("/", "cstool_version") ? f.attribute_string("/", "cstool_version") : std::string();

    // material::create (source/core/material.inl:25-34)
    m.barrier = float(as_double(div(property(f, "barrier"), kEV), "barrier"));

    // kieft_elastic::create (source/physics/kieft/elastic.h:120-166)
    if (!f.exists("/kieft/elastic"))
        throw std::runtime_error("Kieft elastic model not found in material file " + filename);
    load_log_imfp(f, "/kieft/elastic/imfp", &m.el_imfp);
    {
        const std::string path = "/kieft/elastic/costheta_icdf";
        m.el_icdf = read_table2d(f, path);
        const Axis K = dimscale(f, path, 0, m.el_icdf.width, true);
        const Axis P = dimscale(f, path, 1, m.el_icdf.height, false);
        set_scale(m.el_icdf, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(P.front()), float(P.back()));
        for (auto& v : m.el_icdf.data) v = std::max(-1.0f, std::min(1.0f, v));
    }
    m.phonon_loss = float(as_double(div(property(f, "phonon_loss"), kEV), "phonon_loss"));
    {
        const Quantity g = unit_table().at("g");
        Quantity me = g;
        me.value = g.value * 9.109383e-28;
        me.value = me.value * 2;
        const Quantity r = div(me, property(f, "effective_A"));
        m.recoil_const = 2 * float(as_double(r, "effective_A"));
    }

    const Quantity fermi_q = property(f, "fermi");
    m.fermi = float(as_double(div(fermi_q, kEV), "fermi"));
    if (f.has_attribute("/", "band_gap"))
        m.band_gap = float(as_double(div(property(f, "band_gap"), kEV), "band_gap"));
    else
        m.band_gap = float(-1.0 * kEV.value / kEV.value);
    m.has_penn = f.exists("/full_penn");
    m.has_kieft_inelastic = f.exists("kieft/inelastic");
    if (!m.has_kieft_inelastic && !m.has_penn)
        throw std::runtime_error("No inelastic model (Kieft or full Penn) found in material file " + filename);
    if (m.has_penn) load_penn(f, fermi_q, &m);
    if (!m.has_kieft_inelastic) return m;

    // kieft_inelastic::create (source/physics/kieft/inelastic.h:212-327)
    load_log_imfp(f, "/kieft/inelastic/imfp", &m.in_imfp);
    {
        const std::string path = "/kieft/inelastic/w0_icdf";
        m.in_icdf = read_table2d(f, path);
        const Axis K = dimscale(f, path, 0, m.in_icdf.width, true);
        const Axis P = dimscale(f, path, 1, m.in_icdf.height, false);
        set_scale(m.in_icdf, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(P.front()), float(P.back()));
        const float unit = float(as_double(div(dataset_unit(f, path), kEV), path + " units"));
        for (int x = 0; x < m.in_icdf.width; ++x) {
            const double K_x = K.at(size_t(x));
            for (int y = 0; y < m.in_icdf.height; ++y) {
                float& v = m.in_icdf.data[size_t(x) * m.in_icdf.height + y];
                const double a = (K_x - fermi_q.value) / kEV.value;
                const double b = double(v * unit);
                v = float(std::log(std::max(0.0, std::min<double>(a, b))));
            }
        }
    }
    {
        const std::string path = "/kieft/ionization/binding_icdf";
        Table2D& t = m.ionisation;
        t = read_table2d(f, path);
        const Axis K = dimscale(f, path, 0, t.width, true);
        const Axis P = dimscale(f, path, 1, t.height, false);
        set_scale(t, float(std::log(K.front() / kEV.value)), float(std::log(K.back() / kEV.value)),
                  float(P.front()), float(P.back()));
        std::vector<double> outer_shells;
        {
            const std::string spath = "/kieft/ionization/outer_shells";
            std::vector<uint64_t> dims;
            auto vals = f.read_dataset(spath, &dims);
            const Quantity u = dataset_unit(f, spath);
            if (!same_dim(u, kEV)) throw std::runtime_error("outer_shells: energy unit expected");
            for (double v : vals) {
                const double q = u.value * v;
                if (q < 100 * kEV.value) outer_shells.push_back(q);
            }
            std::sort(outer_shells.begin(), outer_shells.end());
        }
        const Quantity unit = dataset_unit(f, path);
        if (!same_dim(unit, kEV)) throw std::runtime_error("binding_icdf: energy unit expected");
        // In-place rebuild, reading the partially rebuilt table through
        // get_rounddown exactly as the reference does.
        for (int x = 0; x < t.width; ++x) {
            const double K_x = K.at(size_t(x));
            for (int y = 0; y < t.height; ++y) {
                const float Pv = float(P.at(size_t(y)));
                const double margin = 10 * kEV.value;
                double binding = -1 * kEV.value;
                if (K_x > 100 * kEV.value) {
                    binding = unit.value * double(table2d_get_rounddown(t, float(std::log((K_x + margin) / kEV.value)), Pv));
                    if (binding < 50 * kEV.value || !std::isfinite(binding)) binding = -1 * kEV.value;
                }
                if (binding < 0 * kEV.value) {
                    auto it = std::lower_bound(outer_shells.rbegin(), outer_shells.rend(), K_x, std::greater<double>());
                    if (it != outer_shells.rend()) binding = *it;
                }
                t.data[size_t(x) * t.height + y] = float(binding / kEV.value);
            }
        }
    }
    return m;
}

}  // namespace nbx
