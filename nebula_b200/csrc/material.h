// Material tables for the Kieft & Bosch physics (and the full Penn inelastic
// model when the file has it), loaded from a Nebula .mat file.
//
// The table transforms mirror the reference loaders exactly (same float/double
// operations in the same order), so the device tables are bit-identical to the
// ones the reference CPU path builds:
//   * source/core/material.inl:25-34            barrier
//   * source/physics/kieft/elastic.h:120-166     log-IMFP, clamped cos(theta) ICDF,
//                                                phonon loss, recoil constant
//   * source/physics/kieft/inelastic.h:212-327   log-IMFP, log omega' ICDF,
//                                                rebuilt ionisation table
//   * source/physics/full_penn.h:296-392         log-IMFP, log omega ICDF, q ICDF,
//                                                3-D ionisation table
//   * source/io/hdf5_file.cpp:269-375            3-D tables, axis reconstruction and units
#pragma once

#include <string>
#include <vector>

namespace nbx {

// util::table_1D (source/common/util/table_1D.h): x_index = (x - x_min) * x_step.
struct Table1D {
    int n = 0;
    float x_min = 0, x_step = 0;
    std::vector<float> data;
    float get_scalemax() const { return x_min + (n - 1) / x_step; }
};

// util::table_2D, row-major data[x * height + y] (source/common/util/table_2D.h).
struct Table2D {
    int width = 0, height = 0;
    float x_min = 0, x_step = 0, y_min = 0, y_step = 0;
    std::vector<float> data;
    float at(int x, int y) const { return data[size_t(x) * height + y]; }
};

// util::table_3D, data[(x * height + y) * depth + z] (source/common/util/table_3D.inl:66-70).
struct Table3D {
    int width = 0, height = 0, depth = 0;
    float x_min = 0, x_step = 0, y_min = 0, y_step = 0, z_min = 0, z_step = 0;
    std::vector<float> data;
};

struct MaterialTables {
    std::string filename, name, cstool_version;
    float barrier = 0;
    // kieft_elastic
    Table1D el_imfp;          // log(imfp * nm) vs log(E / eV)
    Table2D el_icdf;          // cos(theta) vs (log E, P)
    float phonon_loss = 0;
    float recoil_const = 0;
    // kieft_inelastic
    Table1D in_imfp;          // log(imfp * nm) vs log(E / eV)
    Table2D in_icdf;          // log(omega' / eV) vs (log E, P)
    Table2D ionisation;       // binding / eV vs (log omega', P), use rounddown
    float fermi = 0;
    float band_gap = -1;
    bool has_kieft_inelastic = false;
    // full_penn (source/physics/full_penn.h:296-392), when the file has it
    bool has_penn = false;
    Table1D penn_imfp;        // log(imfp * nm) vs log(E / eV)
    Table2D penn_omega_icdf;  // log(omega / eV) vs (log E, P)
    Table3D penn_q_icdf;      // hbar q / sqrt(2m) in eV^1/2 vs (log E, omega / E, P)
    Table3D penn_ionisation;  // binding / eV (-1: none) vs (log E, log(omega / E), P), use rounddown
    // min over the mechanisms of exp(imfp scale max), for the Kieft or the
    // full Penn inelastic model
    float max_energy(bool penn = false) const;
};

// Dimensioned unit value in Nebula's unit system (eV, nm, ns, K, e), as parsed
// by source/common/units/unit_parser.h.
struct Quantity {
    double value = 1;
    int dim[5] = {0, 0, 0, 0, 0};   // energy, length, time, temperature, charge
    bool dimensionless() const;
};
Quantity parse_unit(const std::string& text);   // throws on unknown units

MaterialTables load_material(const std::string& filename);   // throws std::runtime_error

// table_2D::get_rounddown (source/common/util/table_2D.inl:97-104), host side.
float table2d_get_rounddown(const Table2D& t, float x, float y);

}  // namespace nbx
