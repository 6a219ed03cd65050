// scenario.cpp — host-side model construction (C++17).
//
// Restates the reference's mesh generator and vehicle scenario builders so
// that a model built here is node-for-node, face-for-face the model crushrs
// builds (see include/crush_scenario.h for the reference functions covered).
// Model construction is host work at set-up; the per-step path is on the GPU.
#include "crush_scenario.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "errors.hpp"

namespace {

enum BlockFace { XMin = 1, XMax = 2, YMin = 4, YMax = 8, ZMin = 16, ZMax = 32 };

struct ContactDef {
    std::vector<uint32_t> nodes;
    std::vector<double> scale;
    std::vector<uint32_t> faces;  // 4 per face
    double stiffness = 0.0, max_distance = 0.0;
};
struct VehicleDef {
    std::vector<uint32_t> nodes;
    uint32_t accel = 0;
    std::vector<uint32_t> front;
    uint32_t frame[3] = {0, 0, 0};  // body-fixed frame of the accelerometer: origin, x axis, plane
};

}  // namespace

struct crush_model {
    std::vector<double> positions;
    std::vector<uint32_t> hexes;
    std::vector<int32_t> hex_part;
    std::vector<std::string> part_names;
    std::vector<crush_material> materials;
    std::vector<double> velocity;
    std::vector<uint32_t> fixed;
    std::vector<std::array<uint32_t, 4>> faces;
    std::vector<std::vector<size_t>> face_set_list;  // in creation order
    std::map<std::string, size_t> face_set_index;
    std::map<std::string, std::vector<uint32_t>> node_sets;
    std::vector<ContactDef> contacts;
    std::vector<VehicleDef> vehicles;
    crush_settings settings;
    // descriptor views
    std::vector<crush_contact> contact_desc;
    std::vector<crush_vehicle> vehicle_desc;
};

namespace {

crush_material elastic_material(double e, double nu, double rho) {
    crush_material m;
    std::memset(&m, 0, sizeof(m));
    m.model = CRUSH_MAT_ELASTIC;
    m.youngs_modulus = e;
    m.poisson_ratio = nu;
    m.density = rho;
    m.transverse_factor = 1.0;
    return m;
}

size_t add_part(crush_model* m, const std::string& name) {
    m->part_names.push_back(name);
    m->materials.push_back(elastic_material(1.0, 0.0, 1.0));  // Model::new default, src/model.rs:170
    return m->part_names.size() - 1;
}

int part_index(const crush_model* m, const std::string& name) {
    for (size_t p = 0; p < m->part_names.size(); ++p)
        if (m->part_names[p] == name) return (int)p;
    return -1;
}

// Mesh::add_hex_block_n, src/mesh.rs:117-171. surfaces: (face bit, set name) in order.
size_t add_hex_block_n(crush_model* m, const std::string& part_name, const double origin[3], const double size[3],
                       const int32_t n_in[3], const std::vector<std::pair<int, std::string>>& surfaces) {
    size_t n[3];
    for (int a = 0; a < 3; ++a) n[a] = (size_t)std::max<int32_t>(n_in[a], 1);
    double d[3];
    for (int a = 0; a < 3; ++a) d[a] = size[a] / (double)n[a];
    size_t node0 = m->positions.size() / 3;
    auto id = [&](size_t i, size_t j, size_t k) { return (uint32_t)(node0 + i + (n[0] + 1) * (j + (n[1] + 1) * k)); };
    for (size_t k = 0; k <= n[2]; ++k)
        for (size_t j = 0; j <= n[1]; ++j)
            for (size_t i = 0; i <= n[0]; ++i) {
                m->positions.push_back(origin[0] + (double)i * d[0]);
                m->positions.push_back(origin[1] + (double)j * d[1]);
                m->positions.push_back(origin[2] + (double)k * d[2]);
                m->velocity.insert(m->velocity.end(), {0.0, 0.0, 0.0});
            }
    size_t part = add_part(m, part_name);
    for (size_t k = 0; k < n[2]; ++k)
        for (size_t j = 0; j < n[1]; ++j)
            for (size_t i = 0; i < n[0]; ++i) {
                uint32_t h[8] = {id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k),
                                 id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)};
                m->hexes.insert(m->hexes.end(), h, h + 8);
                m->hex_part.push_back((int32_t)part);
            }
    for (const auto& sf : surfaces) {
        int a;
        bool max_side;
        switch (sf.first) {
            case XMin: a = 0; max_side = false; break;
            case XMax: a = 0; max_side = true; break;
            case YMin: a = 1; max_side = false; break;
            case YMax: a = 1; max_side = true; break;
            case ZMin: a = 2; max_side = false; break;
            default: a = 2; max_side = true; break;
        }
        int b = (a + 1) % 3, c = (a + 2) % 3;
        size_t fixed = max_side ? n[a] : 0;
        auto at = [&](size_t ib, size_t ic) {
            size_t ijk[3];
            ijk[a] = fixed;
            ijk[b] = ib;
            ijk[c] = ic;
            return id(ijk[0], ijk[1], ijk[2]);
        };
        std::vector<size_t> set;
        for (size_t ic = 0; ic < n[c]; ++ic)
            for (size_t ib = 0; ib < n[b]; ++ib) {
                uint32_t p0 = at(ib, ic), p1 = at(ib + 1, ic), p2 = at(ib + 1, ic + 1), p3 = at(ib, ic + 1);
                if (max_side) m->faces.push_back({p0, p1, p2, p3});
                else m->faces.push_back({p0, p3, p2, p1});
                set.push_back(m->faces.size() - 1);
            }
        m->face_set_index[sf.second] = m->face_set_list.size();
        m->face_set_list.push_back(set);
    }
    std::vector<uint32_t> all;
    for (size_t i = node0; i < m->positions.size() / 3; ++i) all.push_back((uint32_t)i);
    m->node_sets[part_name] = all;
    return part;
}

// Mesh::add_hex_block, src/mesh.rs:111 (n = round(size / h), at least 1; f64::round rounds half away from zero).
size_t add_hex_block(crush_model* m, const std::string& part_name, const double origin[3], const double size[3], double h,
                     const std::vector<std::pair<int, std::string>>& surfaces) {
    int32_t n[3];
    for (int a = 0; a < 3; ++a) n[a] = (int32_t)std::max(std::round(size[a] / h), 1.0);
    return add_hex_block_n(m, part_name, origin, size, n, surfaces);
}

const std::vector<size_t>* face_set(const crush_model* m, const std::string& name) {
    auto it = m->face_set_index.find(name);
    return it == m->face_set_index.end() ? nullptr : &m->face_set_list[it->second];
}

// Mesh::face_set_nodes, src/mesh.rs:97 (sorted, unique).
bool face_set_nodes(const crush_model* m, const std::string& name, std::vector<uint32_t>* out) {
    const std::vector<size_t>* set = face_set(m, name);
    if (!set) return false;
    std::set<uint32_t> s;
    for (size_t f : *set) s.insert(m->faces[f].begin(), m->faces[f].end());
    out->assign(s.begin(), s.end());
    return true;
}

// Mesh::part_nodes, src/mesh.rs:74.
std::vector<uint32_t> part_nodes(const crush_model* m, int part) {
    std::set<uint32_t> s;
    for (size_t e = 0; e < m->hex_part.size(); ++e)
        if (m->hex_part[e] == part) s.insert(&m->hexes[8 * e], &m->hexes[8 * e] + 8);
    return std::vector<uint32_t>(s.begin(), s.end());
}

// Material::scaled, src/material.rs:200.
crush_material scaled(const crush_material& in, double f) {
    crush_material m = in;
    m.youngs_modulus *= f;
    m.density *= f;
    m.yield_stress *= f;
    m.hardening *= f;
    for (int i = 0; i < m.n_curve; ++i) m.curve[i][1] *= f;
    if (m.has_densification) m.densification[1] *= f;
    return m;
}

struct VehicleCtx {
    const crush_vehicle_spec* spec;
    std::string name;
    double y_center, z_bottom;
};

double frontal_area(const crush_vehicle_spec& v) { return v.size[1] * v.size[2]; }
double contact_modulus(const crush_vehicle_spec& v) {
    return v.contact_modulus > 0.0 ? v.contact_modulus : v.material.youngs_modulus;
}
// Vehicle::has_crush_zone, src/vehicle.rs:323 (a length of 0 means the whole block).
bool has_crush_zone(const crush_vehicle_spec& v) { return v.crush_zone_length > 0.0 && v.crush_zone_length < v.size[0] - 1e-9; }
double bumper_thickness(const crush_vehicle_spec& v) { return has_crush_zone(v) && v.bumper[0] > 0.0 ? v.bumper[0] : 0.0; }
double bumper_mass(const crush_vehicle_spec& v) { return bumper_thickness(v) > 0.0 ? v.bumper[1] : 0.0; }
// Vehicle::honeycomb_length, src/vehicle.rs:374.
double honeycomb_length(const crush_vehicle_spec& v) { return v.crush_zone_length - bumper_thickness(v); }
double block_density(const crush_vehicle_spec& v) { return v.mass / (v.size[0] * v.size[1] * v.size[2]); }
// Vehicle::crush_density / body_density, src/vehicle.rs:454-467.
double crush_density(const crush_vehicle_spec& v) {
    if (v.crush_zone_mass > 0.0 && has_crush_zone(v)) return (v.crush_zone_mass - bumper_mass(v)) / (honeycomb_length(v) * frontal_area(v));
    return block_density(v);
}
double body_density(const crush_vehicle_spec& v) {
    if (v.crush_zone_mass > 0.0 && has_crush_zone(v))
        return (v.mass - v.crush_zone_mass) / ((v.size[0] - v.crush_zone_length) * frontal_area(v));
    return block_density(v);
}
// Vehicle::contact_stiffness_per_node, src/vehicle.rs:384: the crush zone's
// element length at the front when there is a crush zone.
double contact_stiffness_per_node(const crush_vehicle_spec& v, size_t n_face, double h) {
    const double h_front = has_crush_zone(v) && v.crush_element_size > 0.0 ? v.crush_element_size : h;
    return contact_modulus(v) * frontal_area(v) / ((double)n_face * h_front);
}
bool in_rail_box(const crush_vehicle_spec& v, double y, double z) {
    return v.has_rail_box && std::fabs(y) < 0.5 * v.rail_box_width && z > v.rail_box_z[0] && z < v.rail_box_z[1];
}
// Vehicle::rail_box_factors, src/vehicle.rs:367.
void rail_box_factors(const crush_vehicle_spec& v, double area_fraction, double* f_rails, double* f_skin) {
    double f = std::min(std::max(v.has_rail_box ? v.rail_box_force_fraction : 0.0, 0.0), 1.0);
    double a = std::min(std::max(area_fraction, 1e-6), 1.0 - 1e-6);
    *f_rails = f / a;
    *f_skin = (1.0 - f) / (1.0 - a);
}

crush_material crush_material_of(const crush_vehicle_spec& v) {
    crush_material m = v.material;
    if (!(m.density > 0.0)) m.density = crush_density(v);
    return m;
}

// Move the elements of part `from` whose cross-section centroid lies in the
// rail box to a new part `to` (src/vehicle.rs:713-731).
void carve_rail_box(crush_model* m, const VehicleCtx& vc, int from, const std::string& to_name) {
    size_t to = add_part(m, to_name);
    for (size_t e = 0; e < m->hex_part.size(); ++e) {
        if (m->hex_part[e] != from) continue;
        double ys = 0.0, zs = 0.0;
        for (int i = 0; i < 8; ++i) {
            ys += m->positions[3 * m->hexes[8 * e + i] + 1];
            zs += m->positions[3 * m->hexes[8 * e + i] + 2];
        }
        double yc = ys / 8.0 - vc.y_center, zc = zs / 8.0 - vc.z_bottom;
        if (in_rail_box(*vc.spec, yc, zc)) m->hex_part[e] = (int32_t)to;
    }
}

// Mesh::merge_coincident_nodes, src/mesh.rs:176-233: nodes within `tol` of
// an earlier kept node (looked up in its rounded cell and the 26 around it)
// merge into it; the kept nodes are renumbered in order and every element,
// face and node set follows (node sets sorted, duplicates dropped).
size_t merge_coincident_nodes(crush_model* m, double tol) {
    const size_t n = m->positions.size() / 3;
    auto key = [&](const double* p) {
        return std::array<long long, 3>{(long long)std::round(p[0] / tol), (long long)std::round(p[1] / tol), (long long)std::round(p[2] / tol)};
    };
    std::map<std::array<long long, 3>, size_t> first;
    std::vector<uint32_t> map(n, 0);
    std::vector<double> kept;
    kept.reserve(3 * n);
    size_t merged = 0;
    for (size_t i = 0; i < n; ++i) {
        const double* p = &m->positions[3 * i];
        const std::array<long long, 3> k = key(p);
        long long found = -1;
        for (int dx = -1; dx <= 1 && found < 0; ++dx)
            for (int dy = -1; dy <= 1 && found < 0; ++dy)
                for (int dz = -1; dz <= 1 && found < 0; ++dz) {
                    auto it = first.find({k[0] + dx, k[1] + dy, k[2] + dz});
                    if (it == first.end()) continue;
                    const double* q = &kept[3 * it->second];
                    if (std::fabs(q[0] - p[0]) <= tol && std::fabs(q[1] - p[1]) <= tol && std::fabs(q[2] - p[2]) <= tol)
                        found = (long long)it->second;
                }
        if (found >= 0) {
            map[i] = (uint32_t)found;
            ++merged;
        } else {
            map[i] = (uint32_t)(kept.size() / 3);
            first[k] = kept.size() / 3;
            kept.insert(kept.end(), p, p + 3);
        }
    }
    if (merged == 0) return 0;
    m->positions = kept;
    m->velocity.assign(kept.size(), 0.0);
    for (uint32_t& x : m->hexes) x = map[x];
    for (auto& f : m->faces)
        for (uint32_t& x : f) x = map[x];
    for (auto& kv : m->node_sets) {
        std::vector<uint32_t> v;
        for (uint32_t x : kv.second) v.push_back(map[x]);
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        kv.second = v;
    }
    for (uint32_t& x : m->fixed) x = map[x];
    return merged;
}

// add_vehicle, src/vehicle.rs:663-748. A homogeneous block (the rail box,
// when asked, is then carved out of the whole block), or the two-part
// vehicle: body block (part <name>), crush-zone block (<name>_crush) and an
// optional one-element bumper layer (<name>_bumper) with matching y/z grids,
// rear to front along the heading, underbody faces merged into
// <name>_bottom, the rail box carved out of the crush zone and the bumper,
// coincident nodes merged, and node set <name> spanning all the parts.
void add_vehicle(crush_model* m, VehicleCtx& vc, double front_x, bool plus_x, double h) {
    const crush_vehicle_spec& v = *vc.spec;
    double x0 = plus_x ? front_x - v.size[0] : front_x;
    int face = plus_x ? XMax : XMin;
    double origin[3] = {x0, vc.y_center - v.size[1] / 2.0, vc.z_bottom};
    const std::string front = vc.name + "_front", bottom = vc.name + "_bottom";
    if (!has_crush_zone(v)) {
        add_hex_block(m, vc.name, origin, v.size, h, {{face, front}, {ZMin, bottom}});
        if (v.has_rail_box) carve_rail_box(m, vc, part_index(m, vc.name), vc.name + "_rails");
        return;
    }
    const double t_b = bumper_thickness(v);
    const double l_c = v.crush_zone_length - t_b;
    const double l_b = v.size[0] - v.crush_zone_length;
    auto count = [](double len, double step) { return (int32_t)std::max(std::round(len / step), 1.0); };
    const int32_t ny = count(v.size[1], h), nz = count(v.size[2], h), nxb = count(l_b, h);
    const int32_t nxc = count(l_c, v.crush_element_size > 0.0 ? v.crush_element_size : h);
    const double body_x0 = plus_x ? x0 : x0 + l_c + t_b;
    const double crush_x0 = plus_x ? x0 + l_b : x0 + t_b;
    const double bumper_x0 = plus_x ? x0 + l_b + l_c : x0;
    auto sub = [&](const char* part) { return bottom + "_" + part; };
    {
        const double o[3] = {body_x0, origin[1], origin[2]}, sz[3] = {l_b, v.size[1], v.size[2]};
        const int32_t n[3] = {nxb, ny, nz};
        add_hex_block_n(m, vc.name, o, sz, n, {{ZMin, sub("body")}});
    }
    const std::string crush_name = vc.name + "_crush", bumper_name = vc.name + "_bumper";
    std::vector<std::string> names{crush_name}, bottoms{sub("body"), sub("crush")};
    {
        const double o[3] = {crush_x0, origin[1], origin[2]}, sz[3] = {l_c, v.size[1], v.size[2]};
        const int32_t n[3] = {nxc, ny, nz};
        if (t_b > 0.0) add_hex_block_n(m, crush_name, o, sz, n, {{ZMin, sub("crush")}});
        else add_hex_block_n(m, crush_name, o, sz, n, {{face, front}, {ZMin, sub("crush")}});
    }
    if (t_b > 0.0) {
        const double o[3] = {bumper_x0, origin[1], origin[2]}, sz[3] = {t_b, v.size[1], v.size[2]};
        const int32_t n[3] = {1, ny, nz};
        add_hex_block_n(m, bumper_name, o, sz, n, {{face, front}, {ZMin, sub("bumper")}});
        names.push_back(bumper_name);
        bottoms.push_back(sub("bumper"));
    }
    std::vector<size_t> bottom_faces;
    for (const std::string& b : bottoms) {
        auto it = m->face_set_index.find(b);
        if (it == m->face_set_index.end()) continue;
        const std::vector<size_t>& set = m->face_set_list[it->second];
        bottom_faces.insert(bottom_faces.end(), set.begin(), set.end());
        m->face_set_index.erase(it);
    }
    m->face_set_index[bottom] = m->face_set_list.size();
    m->face_set_list.push_back(bottom_faces);
    if (v.has_rail_box) {
        const int crush_part = part_index(m, crush_name), bumper_part = part_index(m, bumper_name);
        carve_rail_box(m, vc, crush_part, vc.name + "_rails");
        if (bumper_part >= 0) carve_rail_box(m, vc, bumper_part, vc.name + "_bumper_rails");
    }
    merge_coincident_nodes(m, 1e-6 * h);
    std::vector<uint32_t> all = m->node_sets[vc.name];
    for (const std::string& nm : names) all.insert(all.end(), m->node_sets[nm].begin(), m->node_sets[nm].end());
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    m->node_sets[vc.name] = all;
}

void set_velocity(crush_model* m, const std::string& set, const double v[3]) {
    for (uint32_t n : m->node_sets[set])
        for (int d = 0; d < 3; ++d) m->velocity[3 * n + d] = v[d];
}

// assign_vehicle, src/vehicle.rs:750-790: materials (the rail box and the
// skin of the crush zone scaled by rail_box_factors over their element
// counts; a two-part vehicle's elastic body and bumper plate) and the
// initial velocity of node set <name>.
void assign_vehicle(crush_model* m, const VehicleCtx& vc, const double vel[3]) {
    const crush_vehicle_spec& v = *vc.spec;
    crush_material crush = crush_material_of(v);
    const bool two_part = has_crush_zone(v) && part_index(m, vc.name + "_crush") >= 0;
    if (two_part) m->materials[part_index(m, vc.name)] = elastic_material(v.body_modulus, 0.3, body_density(v));
    int skin = part_index(m, two_part ? vc.name + "_crush" : vc.name);
    int rails = v.has_rail_box ? part_index(m, vc.name + "_rails") : -1;
    double fr = 1.0, fs = 1.0;
    if (rails >= 0) {
        size_t n_rails = 0, n_skin = 0;
        for (int32_t p : m->hex_part) {
            n_rails += p == rails;
            n_skin += p == skin;
        }
        if (n_rails > 0 && n_skin > 0) rail_box_factors(v, (double)n_rails / (double)(n_rails + n_skin), &fr, &fs);
        m->materials[rails] = scaled(crush, fr);
        m->materials[skin] = scaled(crush, fs);
    } else {
        m->materials[skin] = two_part ? scaled(crush, fs) : crush;
    }
    if (two_part && bumper_thickness(v) > 0.0) {
        const crush_material plate = elastic_material(v.bumper[2], 0.3, v.bumper[1] / (v.bumper[0] * frontal_area(v)));
        const int bumper = part_index(m, vc.name + "_bumper"), bumper_rails = part_index(m, vc.name + "_bumper_rails");
        if (bumper >= 0) m->materials[bumper] = scaled(plate, fs);
        if (bumper_rails >= 0) m->materials[bumper_rails] = scaled(plate, fr);
    }
    set_velocity(m, vc.name, vel);
}

// Vehicle::front_contact_scales, src/vehicle.rs:397.
std::vector<double> front_contact_scales(const crush_model* m, const VehicleCtx& vc, double h) {
    const crush_vehicle_spec& v = *vc.spec;
    std::vector<double> out;
    if (!v.has_rail_box) return out;
    std::vector<uint32_t> nodes;
    if (!face_set_nodes(m, vc.name + "_front", &nodes)) return out;
    size_t ny = (size_t)std::max(std::round(v.size[1] / h), 1.0);
    size_t nz = (size_t)std::max(std::round(v.size[2] / h), 1.0);
    double dy = v.size[1] / (double)ny, dz = v.size[2] / (double)nz;
    double lo[3] = {1e308, 1e308, 1e308}, hi[3] = {-1e308, -1e308, -1e308};
    for (uint32_t n : nodes)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], m->positions[3 * n + d]);
            hi[d] = std::max(hi[d], m->positions[3 * n + d]);
        }
    double y_center = 0.5 * (lo[1] + hi[1]), z_bottom = lo[2];
    size_t cells = ny * nz, n_rails = 0;
    for (size_t c = 0; c < cells; ++c)
        if (in_rail_box(v, (double)(c % ny) * dy + 0.5 * dy - 0.5 * v.size[1], (double)(c / ny) * dz + 0.5 * dz)) ++n_rails;
    if (n_rails == 0 || n_rails == cells) return out;
    double fr, fs;
    rail_box_factors(v, (double)n_rails / (double)cells, &fr, &fs);
    static const double S[4][2] = {{-0.5, -0.5}, {0.5, -0.5}, {-0.5, 0.5}, {0.5, 0.5}};
    for (uint32_t n : nodes) {
        const double* p = &m->positions[3 * n];
        double sum = 0.0;
        int count = 0;
        for (const auto& s : S) {
            double yc = p[1] - y_center + s[0] * dy, zc = p[2] - z_bottom + s[1] * dz;
            if (std::fabs(yc) < 0.5 * v.size[1] && zc > 0.0 && zc < v.size[2]) {
                sum += in_rail_box(v, yc, zc) ? fr : fs;
                ++count;
            }
        }
        out.push_back(count > 0 ? sum / (double)count : 1.0);
    }
    return out;
}

// add_ground, src/vehicle.rs:829 (a fixed elastic slab, face set `<name>_face`).
void add_ground(crush_model* m, double z, const double x[2], const double y[2], double thickness) {
    double h = std::max(std::min(x[1] - x[0], y[1] - y[0]) / 8.0, thickness);
    double origin[3] = {x[0], y[0], z - thickness};
    double size[3] = {x[1] - x[0], y[1] - y[0], thickness};
    add_hex_block(m, "ground", origin, size, h, {{ZMax, "ground_face"}});
}

void add_contact_one_way(crush_model* m, const std::string& nodes_set, const std::string& faces_set, double k, double md,
                         const std::vector<double>& scale) {
    ContactDef c;
    face_set_nodes(m, nodes_set, &c.nodes);
    for (size_t f : *face_set(m, faces_set)) c.faces.insert(c.faces.end(), m->faces[f].begin(), m->faces[f].end());
    c.stiffness = k;
    c.max_distance = md;
    c.scale = scale;
    m->contacts.push_back(c);
}

// add_ground_contact, src/vehicle.rs:838. `n_face_override` (> 0) reproduces
// the T-bone side profile, whose `<name>_front` set does not exist so the
// reference falls back to the number of underbody nodes.
void add_ground_contact(crush_model* m, const VehicleCtx& vc, double clearance, double h, bool side_profile) {
    std::vector<uint32_t> bottom, front;
    face_set_nodes(m, vc.name + "_bottom", &bottom);
    size_t n_bottom = bottom.empty() ? 1 : bottom.size();
    size_t n_face = (!side_profile && face_set_nodes(m, vc.name + "_front", &front)) ? front.size() : n_bottom;
    int g = part_index(m, "ground");
    m->materials[g] = elastic_material(1e9, 0.3, 1000.0);
    for (uint32_t n : m->node_sets["ground"]) m->fixed.push_back(n);
    add_contact_one_way(m, vc.name + "_bottom", "ground_face", contact_stiffness_per_node(*vc.spec, n_face, h), clearance + 0.3, {});
}

// Model::add_contact_pair_scaled, src/model.rs:257.
void add_contact_pair_scaled(crush_model* m, const std::string& a, const std::string& b, double k, double md,
                             const std::vector<double>& sa, const std::vector<double>& sb) {
    add_contact_one_way(m, a, b, 0.5 * k, md, sa);
    add_contact_one_way(m, b, a, 0.5 * k, md, sb);
}

// add_vehicle_accelerometer, src/vehicle.rs:792-822 -> Mesh::nearest_node (first minimum).
uint32_t accelerometer_node(const crush_model* m, const std::string& part, const std::string& front_face) {
    int p = part_index(m, part);
    std::vector<uint32_t> nodes = part_nodes(m, p);
    double lo[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    double hi[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    for (uint32_t n : nodes)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], m->positions[3 * n + d]);
            hi[d] = std::max(hi[d], m->positions[3 * n + d]);
        }
    std::vector<uint32_t> front;
    face_set_nodes(m, front_face, &front);
    double c[3] = {0, 0, 0};
    for (uint32_t n : front)
        for (int d = 0; d < 3; ++d) c[d] += m->positions[3 * n + d] / (double)front.size();
    double at[3] = {0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), lo[2] + 0.35 * (hi[2] - lo[2])};
    for (int d = 0; d < 2; ++d) {
        double len = hi[d] - lo[d];
        if (c[d] <= lo[d] + 1e-6 * len) at[d] = hi[d] - 0.25 * len;
        else if (c[d] >= hi[d] - 1e-6 * len) at[d] = lo[d] + 0.25 * len;
    }
    uint32_t best = nodes.empty() ? 0 : nodes[0];
    double best_d = 1e308;
    bool first = true;
    for (uint32_t n : nodes) {
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) d2 += (m->positions[3 * n + d] - at[d]) * (m->positions[3 * n + d] - at[d]);
        if (first || d2 < best_d) { best = n; best_d = d2; first = false; }
    }
    return best;
}

// Mesh::min_edge_at, src/mesh.rs:236-249: the shortest hexahedron edge at `node`.
double min_edge_at(const crush_model* m, uint32_t node) {
    static const int EDGES[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    double best = 1.0 / 0.0;
    for (size_t e = 0; e < m->hex_part.size(); ++e) {
        const uint32_t* h = &m->hexes[8 * e];
        if (std::find(h, h + 8, node) == h + 8) continue;
        for (const auto& ed : EDGES) {
            if (h[ed[0]] != node && h[ed[1]] != node) continue;
            const double* p = &m->positions[3 * h[ed[0]]];
            const double* q = &m->positions[3 * h[ed[1]]];
            const double d = std::sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]));
            best = std::min(best, d);
        }
    }
    return best;
}

// Mesh::best_aligned_neighbour, src/mesh.rs:265-288: among the part's nodes
// within `radius` of `node` (not `node`, not excluded), the one whose
// direction has the largest cosine with `dir` (first maximum).
bool best_aligned_neighbour(const crush_model* m, uint32_t node, const double dir[3], double radius, const std::vector<uint32_t>& cand,
                            long long exclude, uint32_t* out, double* cos_out) {
    const double* o = &m->positions[3 * node];
    const double dn = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    bool found = false;
    double best = 0.0;
    for (uint32_t n : cand) {
        if (n == node || (long long)n == exclude) continue;
        const double r[3] = {m->positions[3 * n] - o[0], m->positions[3 * n + 1] - o[1], m->positions[3 * n + 2] - o[2]};
        const double rn = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        if (rn > radius || rn == 0.0) continue;
        const double c = (r[0] * dir[0] + r[1] * dir[1] + r[2] * dir[2]) / (rn * dn);
        if (!found || c > best) {
            found = true;
            best = c;
            *out = n;
        }
    }
    *cos_out = best;
    return found;
}

// Model::add_accelerometer_at, src/model.rs:185-214: the body-fixed frame
// of accelerometer node `rec` in part `part`: x axis towards the neighbour
// best aligned with +X (else the origin moves to the -X neighbour), plane
// node the origin's neighbour towards +Y (else -Y), within 1.75 x the
// shortest edge at `rec`.
void accelerometer_frame(const crush_model* m, const std::string& part, uint32_t rec, uint32_t frame[3]) {
    const std::vector<uint32_t> cand = part_nodes(m, part_index(m, part));
    const double radius = 1.75 * min_edge_at(m, rec);
    uint32_t origin = rec, x_axis = rec, n = 0;
    double c = 0.0;
    const double px[3] = {1.0, 0.0, 0.0}, mx[3] = {-1.0, 0.0, 0.0}, py[3] = {0.0, 1.0, 0.0}, my[3] = {0.0, -1.0, 0.0};
    if (best_aligned_neighbour(m, rec, px, radius, cand, -1, &n, &c) && c > 0.5) x_axis = n;
    else if (best_aligned_neighbour(m, rec, mx, radius, cand, -1, &n, &c)) origin = n;
    uint32_t plane = origin;
    if (best_aligned_neighbour(m, origin, py, radius, cand, x_axis, &n, &c) && c > 0.5) plane = n;
    else if (best_aligned_neighbour(m, origin, my, radius, cand, x_axis, &n, &c)) plane = n;
    frame[0] = origin;
    frame[1] = x_axis;
    frame[2] = plane;
}

void add_vehicle_output(crush_model* m, const std::string& name, const std::string& front_face) {
    VehicleDef v;
    v.nodes = m->node_sets[name];
    v.accel = accelerometer_node(m, name, front_face);
    face_set_nodes(m, front_face, &v.front);
    accelerometer_frame(m, name, v.accel, v.frame);
    m->vehicles.push_back(v);
}

int check_spec(const crush_vehicle_spec& v) {
    if (!(v.mass > 0.0) || !(v.size[0] > 0.0) || !(v.size[1] > 0.0) || !(v.size[2] > 0.0))
        return crush::fail(CRUSH_ERR_INVALID, "a vehicle needs a positive mass and size");
    if (v.material.model != CRUSH_MAT_HONEYCOMB) return crush::fail(CRUSH_ERR_UNSUPPORTED, "vehicle crush material must be honeycomb");
    if (!(v.material.youngs_modulus > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "vehicle modulus must be positive");
    if (has_crush_zone(v)) {
        if (!(v.body_modulus > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "a crush zone needs a positive body modulus");
        if (v.crush_zone_mass > 0.0 && !(v.crush_zone_mass < v.mass)) return crush::fail(CRUSH_ERR_INVALID, "crush zone mass must be below the vehicle mass");
        if (v.bumper[0] > 0.0 && (!(v.bumper[0] < v.crush_zone_length) || !(v.bumper[1] > 0.0) || !(v.bumper[2] > 0.0)))
            return crush::fail(CRUSH_ERR_INVALID, "a bumper needs thickness below the crush zone length, a positive mass and modulus");
        if (v.crush_zone_mass > 0.0 && !(v.crush_zone_mass > bumper_mass(v)))
            return crush::fail(CRUSH_ERR_INVALID, "crush zone mass must exceed the bumper mass");
    }
    return CRUSH_OK;
}

}  // namespace

extern "C" {

crush_settings crush_settings_default(double end_time) {
    crush_settings s;
    std::memset(&s, 0, sizeof(s));
    s.end_time = end_time;
    s.dt_scale = 0.85;
    s.time_step = 0.0;
    s.adaptive_check_steps = 5;
    s.hourglass = 0.1;
    s.velocity_damping = 1.0;
    s.mass_scaling = 0.25;
    s.stop_rule = CRUSH_STOP_END_TIME;
    s.max_steps = 0;
    return s;
}

int crush_scenario_build(const crush_scenario* s, crush_model** out) {
    if (!s || !out) return crush::fail(CRUSH_ERR_INVALID, "null scenario");
    *out = nullptr;
    int st = check_spec(s->a);
    if (st == CRUSH_OK && s->layout != CRUSH_LAYOUT_BARRIER) st = check_spec(s->b);
    if (st != CRUSH_OK) return st;
    if (!(s->element_size > 0.0)) return crush::fail(CRUSH_ERR_INVALID, "element size must be positive");
    crush_model* m = new crush_model();
    const double h = s->element_size, gap = 0.005;
    VehicleCtx a{&s->a, "a", 0.0, 0.0};
    VehicleCtx b{&s->b, "b", s->layout == CRUSH_LAYOUT_TBONE ? -s->offset : s->offset, 0.0};
    bool road = s->clearance >= 0.0;
    if (s->layout == CRUSH_LAYOUT_HEADON) {
        // HeadOn::build, src/headon.rs:40-66
        add_vehicle(m, a, -gap, true, h);
        add_vehicle(m, b, gap, false, h);
        if (road) {
            double w = std::max(s->a.size[1], s->b.size[1]) + 2.0 * std::fabs(s->offset);
            double xr[2] = {-s->a.size[0] - 3.0, s->b.size[0] + 3.0}, yr[2] = {-w, w};
            add_ground(m, -s->clearance, xr, yr, 0.3);
        }
        double va[3] = {s->speed_a, 0.0, 0.0}, vb[3] = {-s->speed_b, 0.0, 0.0};
        assign_vehicle(m, a, va);
        assign_vehicle(m, b, vb);
        if (road) {
            add_ground_contact(m, a, s->clearance, h, false);
            add_ground_contact(m, b, s->clearance, h, false);
        }
        std::vector<uint32_t> fa, fb;
        face_set_nodes(m, "a_front", &fa);
        face_set_nodes(m, "b_front", &fb);
        size_t n_face = std::min(fa.size(), fb.size());
        double k = std::min(contact_stiffness_per_node(s->a, n_face, h), contact_stiffness_per_node(s->b, n_face, h));
        add_contact_pair_scaled(m, "a_front", "b_front", k, 0.3, front_contact_scales(m, a, h), front_contact_scales(m, b, h));
    } else if (s->layout == CRUSH_LAYOUT_TBONE) {
        // src/bin/crushrs.rs:550-576: A's front into the x-min side of B.
        add_vehicle(m, a, -gap, true, h);
        double origin[3] = {gap, -s->offset - s->b.size[1] / 2.0, 0.0};
        add_hex_block(m, "b", origin, s->b.size, h, {{XMin, "b_front"}, {ZMin, "b_bottom"}});
        if (road) {
            double w = s->b.size[1] + s->a.size[1];
            double xr[2] = {-s->a.size[0] - 3.0, s->b.size[0] + 3.0}, yr[2] = {-w, w};
            add_ground(m, -s->clearance, xr, yr, 0.3);
        }
        double va[3] = {s->speed_a, 0.0, 0.0}, vb[3] = {0.0, s->speed_b, 0.0};
        assign_vehicle(m, a, va);
        m->materials[part_index(m, "b")] = crush_material_of(s->b);
        set_velocity(m, "b", vb);
        if (road) {
            add_ground_contact(m, a, s->clearance, h, false);
            add_ground_contact(m, b, s->clearance, h, true);
        }
        std::vector<uint32_t> fb;
        face_set_nodes(m, "b_front", &fb);
        double k = std::min(contact_stiffness_per_node(s->b, fb.size(), h), contact_stiffness_per_node(s->a, fb.size(), h));
        add_contact_pair_scaled(m, "a_front", "b_front", k, 0.3, {}, {});
    } else if (s->layout == CRUSH_LAYOUT_BARRIER) {
        // barrier_model, src/vehicle.rs:951-973: A into a fixed elastic wall
        // (add_rigid_wall, :851: face set wall_face at x = 0 facing -x), the
        // road under A, and A's front against the wall at A's per-node
        // penalty stiffness.
        const crush_vehicle_spec& v = s->a;
        add_vehicle(m, a, -gap, true, h);
        const double w = v.size[1], z = v.size[2], thickness = 0.2;
        {
            const double y0 = -w * 0.75, y1 = w * 0.75, z0 = -0.2 * z, z1 = 1.2 * z;
            const double hw = std::max(std::min(y1 - y0, z1 - z0) / 4.0, thickness);
            const double origin[3] = {0.0, y0, z0}, size[3] = {thickness, y1 - y0, z1 - z0};
            add_hex_block(m, "wall", origin, size, hw, {{XMin, "wall_face"}});
        }
        if (road) {
            double xr[2] = {-v.size[0] - 1.0, -0.3}, yr[2] = {-w, w};
            add_ground(m, -s->clearance, xr, yr, 0.3);
        }
        double va[3] = {s->speed_a, 0.0, 0.0};
        assign_vehicle(m, a, va);
        const int wall = part_index(m, "wall");
        m->materials[wall] = elastic_material(1e9, 0.3, 1000.0);
        for (uint32_t n : m->node_sets["wall"]) m->fixed.push_back(n);
        if (road) add_ground_contact(m, a, s->clearance, h, false);
        std::vector<uint32_t> fa;
        face_set_nodes(m, "a_front", &fa);
        add_contact_pair_scaled(m, "a_front", "wall_face", contact_stiffness_per_node(v, fa.size(), h), 0.3, front_contact_scales(m, a, h), {});
    } else {
        delete m;
        return crush::fail(CRUSH_ERR_INVALID, "unknown layout");
    }
    m->settings = s->settings;
    add_vehicle_output(m, "a", "a_front");
    if (s->layout != CRUSH_LAYOUT_BARRIER) add_vehicle_output(m, "b", "b_front");
    *out = m;
    return CRUSH_OK;
}

void crush_model_free(crush_model* m) { delete m; }

int crush_model_vehicle_frame(const crush_model* m, int32_t vehicle, uint32_t frame[3]) {
    if (!m || !frame || vehicle < 0 || vehicle >= (int32_t)m->vehicles.size()) return crush::fail(CRUSH_ERR_INVALID, "no such vehicle");
    for (int k = 0; k < 3; ++k) frame[k] = m->vehicles[vehicle].frame[k];
    return CRUSH_OK;
}

crush_settings* crush_model_settings(crush_model* m) { return m ? &m->settings : nullptr; }

int crush_model_desc_get(const crush_model* mc, crush_model_desc* d) {
    if (!mc || !d) return crush::fail(CRUSH_ERR_INVALID, "null model");
    crush_model* m = const_cast<crush_model*>(mc);
    m->contact_desc.clear();
    for (const ContactDef& c : m->contacts) {
        crush_contact k;
        k.n_nodes = (int64_t)c.nodes.size();
        k.nodes = c.nodes.data();
        k.node_scale = c.scale.empty() ? nullptr : c.scale.data();
        k.n_faces = (int64_t)c.faces.size() / 4;
        k.faces = c.faces.data();
        k.stiffness = c.stiffness;
        k.max_distance = c.max_distance;
        m->contact_desc.push_back(k);
    }
    m->vehicle_desc.clear();
    for (const VehicleDef& v : m->vehicles) {
        crush_vehicle w;
        w.n_nodes = (int64_t)v.nodes.size();
        w.nodes = v.nodes.data();
        w.accel_node = v.accel;
        w.n_front = (int64_t)v.front.size();
        w.front_nodes = v.front.data();
        m->vehicle_desc.push_back(w);
    }
    std::memset(d, 0, sizeof(*d));
    d->n_nodes = (int64_t)m->positions.size() / 3;
    d->positions = m->positions.data();
    d->n_hexes = (int64_t)m->hex_part.size();
    d->hexes = m->hexes.data();
    d->hex_part = m->hex_part.data();
    d->n_parts = (int32_t)m->materials.size();
    d->materials = m->materials.data();
    d->initial_velocity = m->velocity.data();
    d->n_fixed = (int64_t)m->fixed.size();
    d->fixed_nodes = m->fixed.data();
    d->n_contacts = (int32_t)m->contact_desc.size();
    d->contacts = m->contact_desc.data();
    d->n_vehicles = (int32_t)m->vehicle_desc.size();
    d->vehicles = m->vehicle_desc.data();
    d->settings = m->settings;
    return CRUSH_OK;
}

int crush_model_new(crush_model** out) {
    if (!out) return crush::fail(CRUSH_ERR_INVALID, "null output");
    *out = new crush_model();
    (*out)->settings = crush_settings_default(0.15);
    return CRUSH_OK;
}

int crush_model_add_block(crush_model* m, const double origin[3], const double size[3], const int32_t n[3], int32_t surfaces,
                          int32_t* part_out) {
    if (!m) return crush::fail(CRUSH_ERR_INVALID, "null model");
    std::vector<std::pair<int, std::string>> sf;
    static const int ORDER[6] = {XMin, XMax, YMin, YMax, ZMin, ZMax};
    std::string name = "part" + std::to_string(m->part_names.size());
    for (int f : ORDER)
        if (surfaces & f) sf.push_back({f, name + "_face" + std::to_string(f)});
    size_t p = add_hex_block_n(m, name, origin, size, n, sf);
    if (part_out) *part_out = (int32_t)p;
    return CRUSH_OK;
}

int crush_model_face_set(const crush_model* m, int32_t k, int64_t* n_faces, uint32_t* faces) {
    if (!m || k < 0 || k >= (int32_t)m->face_set_list.size()) return crush::fail(CRUSH_ERR_INVALID, "face set out of range");
    const std::vector<size_t>& set = m->face_set_list[k];
    *n_faces = (int64_t)set.size();
    if (faces)
        for (size_t i = 0; i < set.size(); ++i)
            for (int j = 0; j < 4; ++j) faces[4 * i + j] = m->faces[set[i]][j];
    return CRUSH_OK;
}

int crush_model_set_materials(crush_model* m, int32_t n, const crush_material* mats) {
    if (!m || n != (int32_t)m->materials.size()) return crush::fail(CRUSH_ERR_INVALID, "material count must match parts");
    std::copy(mats, mats + n, m->materials.begin());
    return CRUSH_OK;
}

int crush_model_set_velocity(crush_model* m, const double* v) {
    if (!m || !v) return crush::fail(CRUSH_ERR_INVALID, "null velocity");
    std::copy(v, v + m->velocity.size(), m->velocity.begin());
    return CRUSH_OK;
}

}  // extern "C"
