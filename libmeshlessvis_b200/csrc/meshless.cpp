// Particle data model and the ".sph" text format: the reference's
// meshless_vis/meshless.cpp:22-189 behind include/meshless.h, re-implemented.
//
// Format (as the reference reads and writes it): number of datasets; per
// dataset the number of groups; per group "number_of_terms basis_name
// operator parameters"; then all positions (x y z) of all groups, all weights,
// a has_radii flag and, if set, all radii.  Basis names are "sph", "gaussian",
// "wendland_d3_c2", plus "gaussian_decaying" for the appended basis.
#include <fstream>
#include <string>

#include "meshless.h"

extern "C" {

MeshlessDataset get_simple_meshless_dataset(int number_of_terms, Constraint* h_constraints, float* h_radii,
                                            BasisFunctionId basis_function_id) {
    MeshlessDataset ds;
    ds.number_of_groups = 1;
    ds.groups = new Group[1];
    Group& g = ds.groups[0];
    g.number_of_terms = number_of_terms;
    g.d_number_of_terms = 0;
    g.basis_function_id = basis_function_id;
    g.h_constraints = h_constraints;
    g.d_constraints = nullptr;
    g.h_radii = h_radii;
    g.d_radii = nullptr;
    return ds;
}

void delete_meshless_dataset(MeshlessDataset meshless_dataset) {
    for (int i = 0; i < meshless_dataset.number_of_groups; ++i) {
        delete[] meshless_dataset.groups[i].h_constraints;
        delete[] meshless_dataset.groups[i].h_radii;
    }
    delete[] meshless_dataset.groups;
}

void delete_meshless_datasets(MeshlessDataset* meshless_datasets, int number_of_datasets) {
    if (!meshless_datasets) return;
    for (int i = 0; i < number_of_datasets; ++i) delete_meshless_dataset(meshless_datasets[i]);
    delete[] meshless_datasets;
}

int get_number_of_terms(MeshlessDataset* meshless_dataset) {
    int total = 0;
    for (int i = 0; i < meshless_dataset->number_of_groups; ++i) total += meshless_dataset->groups[i].number_of_terms;
    return total;
}

void shift_meshless_dataset(MeshlessDataset* meshless_dataset, float x, float y, float z) {
    for (int g = 0; g < meshless_dataset->number_of_groups; ++g) {
        Group& grp = meshless_dataset->groups[g];
        for (int k = 0; k < grp.number_of_terms; ++k) {
            grp.h_constraints[k].position.x += x;
            grp.h_constraints[k].position.y += y;
            grp.h_constraints[k].position.z += z;
        }
    }
}

void shift_meshless_datasets(MeshlessDataset* meshless_datasets, int number_of_datasets, float x, float y, float z) {
    for (int i = 0; i < number_of_datasets; ++i) shift_meshless_dataset(meshless_datasets + i, x, y, z);
}

static BasisFunctionId basis_from_name(const std::string& name) {
    if (name == "gaussian") return GAUSSIAN;
    if (name == "wendland_d3_c2") return WENDLAND_D3_C2;
    if (name == "gaussian_decaying") return GAUSSIAN_DECAYING;
    return SPH;
}

static const char* basis_name(BasisFunctionId id) {
    switch (id) {
    case GAUSSIAN: return "gaussian";
    case WENDLAND_D3_C2: return "wendland_d3_c2";
    case GAUSSIAN_DECAYING: return "gaussian_decaying";
    default: return "sph";
    }
}

void load_meshless_datasets_from_file(const char* filename, MeshlessDataset** meshless_datasets,
                                      int* number_of_datasets) {
    *meshless_datasets = nullptr;
    *number_of_datasets = 0;
    std::ifstream in(filename);
    int count = 0;
    if (!(in >> count) || count <= 0) return;
    MeshlessDataset* sets = new MeshlessDataset[count];
    for (int i = 0; i < count; ++i) {
        MeshlessDataset& ds = sets[i];
        ds.number_of_groups = 0;
        in >> ds.number_of_groups;
        if (ds.number_of_groups < 0) ds.number_of_groups = 0;
        ds.groups = new Group[ds.number_of_groups];
        for (int g = 0; g < ds.number_of_groups; ++g) {
            Group& grp = ds.groups[g];
            std::string name, op;
            int parameters = 0;
            grp.number_of_terms = 0;
            in >> grp.number_of_terms >> name >> op >> parameters;
            if (grp.number_of_terms < 0) grp.number_of_terms = 0;
            grp.basis_function_id = basis_from_name(name);
            grp.d_number_of_terms = 0;
            grp.d_constraints = nullptr;
            grp.d_radii = nullptr;
            grp.h_radii = nullptr;
        }
        for (int g = 0; g < ds.number_of_groups; ++g) {
            Group& grp = ds.groups[g];
            grp.h_constraints = new Constraint[grp.number_of_terms];
            for (int k = 0; k < grp.number_of_terms; ++k)
                in >> grp.h_constraints[k].position.x >> grp.h_constraints[k].position.y >>
                    grp.h_constraints[k].position.z;
        }
        for (int g = 0; g < ds.number_of_groups; ++g)
            for (int k = 0; k < ds.groups[g].number_of_terms; ++k) in >> ds.groups[g].h_constraints[k].weight;
        int has_radii = 0;
        in >> has_radii;
        for (int g = 0; g < ds.number_of_groups; ++g) {
            Group& grp = ds.groups[g];
            if (has_radii) {
                grp.h_radii = new float[grp.number_of_terms];
                for (int k = 0; k < grp.number_of_terms; ++k) in >> grp.h_radii[k];
            }
        }
    }
    *meshless_datasets = sets;
    *number_of_datasets = count;
}

void save_meshless_datasets_to_file(const char* filename, MeshlessDataset* meshless_datasets, int number_of_datasets) {
    std::ofstream out(filename);
    out.precision(9);
    out << number_of_datasets << "\n";
    for (int i = 0; i < number_of_datasets; ++i) {
        const MeshlessDataset& ds = meshless_datasets[i];
        out << ds.number_of_groups << "\n";
        for (int g = 0; g < ds.number_of_groups; ++g)
            out << ds.groups[g].number_of_terms << " " << basis_name(ds.groups[g].basis_function_id) << " unused 0\n";
        for (int g = 0; g < ds.number_of_groups; ++g)
            for (int k = 0; k < ds.groups[g].number_of_terms; ++k) {
                const float3& p = ds.groups[g].h_constraints[k].position;
                out << p.x << " " << p.y << " " << p.z << "\n";
            }
        for (int g = 0; g < ds.number_of_groups; ++g)
            for (int k = 0; k < ds.groups[g].number_of_terms; ++k) out << ds.groups[g].h_constraints[k].weight << "\n";
        // The reference decides has_radii from the first group of the first
        // dataset (meshless.cpp:178); per dataset, from its own first group.
        const bool has_radii = ds.number_of_groups > 0 && ds.groups[0].h_radii != nullptr;
        out << (has_radii ? 1 : 0) << "\n";
        if (has_radii)
            for (int g = 0; g < ds.number_of_groups; ++g)
                for (int k = 0; k < ds.groups[g].number_of_terms; ++k)
                    out << (ds.groups[g].h_radii ? ds.groups[g].h_radii[k] : 0.0f) << "\n";
    }
}

Constraint* meshless_new_constraints(int number_of_terms) {
    if (number_of_terms < 0) return nullptr;
    return new Constraint[number_of_terms > 0 ? number_of_terms : 1]();
}

float* meshless_new_radii(int number_of_terms) {
    if (number_of_terms < 0) return nullptr;
    return new float[number_of_terms > 0 ? number_of_terms : 1]();
}

}  // extern "C"
