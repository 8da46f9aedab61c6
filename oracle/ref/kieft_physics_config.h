/* Forced-include header (g++ -include) that selects the Kieft & Bosch
 * inelastic model when compiling the reference's own cpu_mt_main.cpp.
 *
 * It defines the include guard of source/physics_config.h first, so the
 * reference file becomes a no-op, and provides the same four aliases with the
 * commented-out Kieft block of source/physics_config.h:27-33 enabled in place
 * of full_penn (source/physics_config.h:21-24).  Elastic and boundary models
 * are unchanged (source/physics_config.h:36-48).  Test infrastructure only. */
#ifndef __PHYSICS_CONFIG_H_
#define __PHYSICS_CONFIG_H_
#include <iostream>
#include "config/config.h"
#include "core/particle.h"
#include "common/util/table_1D.h"
#include "common/util/table_2D.h"
#include "common/util/table_3D.h"
#include "common/util/random.h"
#include "core/material.h"
#include "physics/kieft/inelastic.h"
#include "physics/kieft/elastic.h"
#include "physics/full_penn.h"
#include "physics/boundary_intersect.h"

template<bool gpu_flag>
using inelastic_scatter = nbl::scatter::kieft_inelastic<gpu_flag, true, true, true, true>;
template<bool gpu_flag>
using elastic_scatter = nbl::scatter::kieft_elastic<gpu_flag, true, true>;
using intersect_t = boundary_intersect<true, true, false>;
template<bool gpu_flag>
using scatter_physics = scatter_list<inelastic_scatter<gpu_flag>, elastic_scatter<gpu_flag>>;
#endif
