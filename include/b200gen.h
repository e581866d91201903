/* b200gen: Newton systems of tet meshes generated on the GPU (C ABI, exported
 * by libb200solve.so).
 *
 * The producers' side of the linear-solve path, written straight into device
 * triplet buffers in the conventions b2s_assemble takes (block-upper 3x3
 * triplets, values column-major, duplicates not summed), for a tet mesh at a
 * given state x with kinetic target x_tilde:
 *   * BDF1 kinetic term, lumped masses: one diagonal block m I per vertex,
 *     gradient m (x - x_tilde)
 *     (libuipc src/backends/cuda/finite_element/bdf/finite_element_bdf1_kinetic.cu:45-68);
 *   * stable Neo-Hookean elasticity per tet, Hessian projected to PSD (9x9
 *     Jacobi eigen-decomposition of d2Psi/dF2), scaled by dt^2 vol: 10
 *     upper blocks per tet
 *     (finite_element/constitutions/stable_neo_hookean_3d.cu:20, 252-263, 486);
 *   * ground half-plane barrier b(d^2) = -(d^2 - dhat^2)^2 log(d^2 / dhat^2)
 *     on the listed candidate vertices, one diagonal block each (zero when
 *     d >= dhat), normal +y
 *     (contact_system/contact_models/ipc_vertex_half_plane_contact_function.h:12-60);
 *   * Dirichlet vertices: rows and columns zeroed, diagonal block I, gradient 0
 *     (finite_element/fem_linear_subsystem.cu:36-52).
 * Triplet slots: [n_verts kinetic][10 n_tets elastic][n_ground ground]; the
 * gradient is summed per vertex in the order kinetic, tets by index, ground.
 * All functions return 0 on success, negative on failure
 * (b2gen_last_error for the message). */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b2gen_material
{
    double mu, lambda;  /* Lame parameters [Pa] */
    double rho;         /* density [kg/m^3] */
    double dt;          /* time step [s] */
    double kappa;       /* barrier stiffness [Pa] */
    double dhat;        /* barrier activation distance [m] */
    double ground_y;    /* ground plane height */
} b2gen_material;

typedef struct b2gen_mesh b2gen_mesh;

/* Host arrays: rest positions [n_verts*3], tets [n_tets*4] (positively
 * oriented in the rest shape), fixed flags [n_verts] (may be NULL), ground
 * candidate vertices [n_ground] (may be NULL). The rest volumes, shape
 * gradients, lumped masses and the vertex-to-tet incidence are built once. */
int b2gen_mesh_create(int device, int32_t n_verts, int32_t n_tets, const double* rest, const int32_t* tets,
                      const uint8_t* fixed, int32_t n_ground, const int32_t* ground, const b2gen_material* mat,
                      b2gen_mesh** out);
int b2gen_mesh_destroy(b2gen_mesh* m);
int64_t b2gen_num_triplets(const b2gen_mesh* m);

/* The Newton system at the device state d_x, d_xtilde [n_verts*3]: writes
 * d_rows, d_cols [num_triplets], d_vals [num_triplets*9], d_grad [n_verts*3]
 * (all device memory), queued on `stream` (a cudaStream_t; NULL = the legacy
 * default stream) and waited for. */
int b2gen_system(b2gen_mesh* m, const double* d_x, const double* d_xtilde, int32_t* d_rows, int32_t* d_cols,
                 double* d_vals, double* d_grad, void* stream);

const char* b2gen_last_error(void);

#ifdef __cplusplus
}
#endif
