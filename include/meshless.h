/*
 * meshless.h -- particle data model of the B200 libMeshlessVis drop-in.
 *
 * Same names, struct layouts and signatures as the reference's
 * include/meshless.h (andrewcorrigan/libmeshlessvis), so that code written
 * against the reference compiles and links unchanged against
 * libmeshless_vis.so.  Each declaration cites the reference line it replaces.
 * The one addition to this header is the appended basis GAUSSIAN_DECAYING and
 * two allocation helpers for callers that cannot use C++ new[] (see below).
 */
#ifndef MESHLESS_H_
#define MESHLESS_H_

#include <vector_types.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/meshless.h:30-35; GAUSSIAN_DECAYING is appended (value 3) and has no
 * reference twin: Phi^(r) = exp(-pi r^2).  The reference GAUSSIAN evaluates
 * exp(+pi r^2) (meshless_vis/fourier_transform.cu:43-46) and is kept as is. */
enum BasisFunctionId
{
    SPH,
    GAUSSIAN,
    WENDLAND_D3_C2,
    GAUSSIAN_DECAYING
};
#ifndef __cplusplus
typedef enum BasisFunctionId BasisFunctionId;
#endif

/* include/meshless.h:37-41: 16-byte AoS particle, position then weight. */
typedef struct __align__(16)
{
    float3 position;
    float weight;
} Constraint;

/* include/meshless.h:43-50.  d_number_of_terms is number_of_terms rounded up
 * to a multiple of number_of_partial_sums * block_length, as the reference's
 * registration pads it (meshless_vis/meshless_vis.cu:264-290). */
typedef struct
{
    int number_of_terms, d_number_of_terms;
    BasisFunctionId basis_function_id;

    Constraint *h_constraints, *d_constraints;
    float *h_radii, *d_radii;
} Group;

/* include/meshless.h:52-57 */
typedef struct
{
    Group* groups;
    int number_of_groups;
} MeshlessDataset;

/* include/meshless.h:59; adopts h_constraints / h_radii (allocated with new[],
 * released by delete_meshless_dataset). */
MeshlessDataset get_simple_meshless_dataset(int number_of_terms, Constraint* h_constraints, float* h_radii,
                                            BasisFunctionId basis_function_id);

/* include/meshless.h:61-62 */
void delete_meshless_dataset(MeshlessDataset meshless_dataset);
void delete_meshless_datasets(MeshlessDataset* meshless_datasets, int number_of_datasets);

/* include/meshless.h:64 */
int get_number_of_terms(MeshlessDataset* meshless_dataset);

/* include/meshless.h:66-67 */
void shift_meshless_dataset(MeshlessDataset* meshless_dataset, float x, float y, float z);
void shift_meshless_datasets(MeshlessDataset* meshless_dataset, int number_of_datasets, float x, float y, float z);

/* include/meshless.h:69-70: the reference's ".sph" text format. */
void load_meshless_datasets_from_file(const char* filename, MeshlessDataset** meshless_datasets,
                                      int* number_of_datasets);
void save_meshless_datasets_to_file(const char* filename, MeshlessDataset* meshless_datasets, int number_of_datasets);

/* Additions (no reference twin): arrays allocated with C++ new[], so that C,
 * Python (ctypes) or other FFI callers can build the arrays that
 * get_simple_meshless_dataset adopts and delete_meshless_dataset releases. */
Constraint* meshless_new_constraints(int number_of_terms);
float* meshless_new_radii(int number_of_terms);

#ifdef __cplusplus
}
#endif

#endif /* MESHLESS_H_ */
