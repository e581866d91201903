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

/* The line search after the solve (engine/advance_ipc.cu:487-570), for a tet
 * mesh: the energy whose gradient and Hessian b2gen_system writes
 * (1/2 m |x - x_tilde|^2 + dt^2 vol Psi_SNH + dt^2 kappa b(d^2) of the ground
 * candidates; infinite when a candidate is at or below the plane), summed in a
 * fixed order, at the device state d_x; and the largest step along d_dx before
 * a ground candidate reaches the plane, as the vertex / half-plane trajectory
 * filter computes it (collision_detection/filters/
 * easy_vertex_half_plane_trajectory_filter.cu:81-145: (1 - 0.1) of the time
 * of impact, capped at 1). */
int b2gen_energy(b2gen_mesh* m, const double* d_x, const double* d_xtilde, double* h_energy, void* stream);
int b2gen_ground_toi(b2gen_mesh* m, const double* d_x, const double* d_dx, double* h_alpha, void* stream);

const char* b2gen_last_error(void);

/* ---- cloth (codim-2D) and affine bodies ------------------------------------------
 * Cloth of n_verts vertices and n_tris triangles (host rest positions
 * [n_verts*3], triangles [n_tris*3], lumped masses [n_verts], fixed flags or
 * NULL):
 *   * kinetic: one diagonal block m I per vertex, gradient m (x - x_tilde);
 *   * Baraff-Witkin strain-limiting stretch + shear per triangle, in the rest
 *     triangle's own uv frame, weight rest area x dt^2, 6 upper blocks
 *     (finite_element/constitutions/strain_limiting_baraff_witkin_shell_2d.cu:75-150,
 *      strain_limiting_baraff_witkin_shell_2d.h:33-280);
 *   * discrete-shell bending per interior edge (hinge (opposite min, edge
 *     min, edge max, opposite max), edges in (min, max) order), Gauss-Newton
 *     Hessian, weight dt^2, 10 upper blocks
 *     (finite_element/constitutions/discrete_shell_bending.cu:96-135, 240-300).
 * Triplet slots [n_verts kinetic][6 n_tris][10 n_hinges]; the cloth's block
 * rows start at vertex_offset in the global system (d_x, d_xtilde, d_grad are
 * global vectors). Gradient per vertex: kinetic, triangles by index, hinges
 * by index. */
typedef struct b2gen_shell_material
{
    double stretch, shear, strain_rate; /* Baraff-Witkin stiffnesses (per area) and strain rate */
    double bend;                        /* bending stiffness */
    double dt;                          /* time step [s] */
} b2gen_shell_material;

typedef struct b2gen_shell b2gen_shell;
int b2gen_shell_create(int device, int32_t n_verts, int32_t n_tris, const double* rest, const int32_t* tris,
                       const double* mass, const uint8_t* fixed, const b2gen_shell_material* mat,
                       b2gen_shell** out);
int b2gen_shell_destroy(b2gen_shell* s);
int64_t b2gen_shell_num_triplets(const b2gen_shell* s);
int32_t b2gen_shell_num_hinges(const b2gen_shell* s);
int b2gen_shell_system(b2gen_shell* s, const double* d_x, const double* d_xtilde, int32_t vertex_offset,
                       int32_t* d_rows, int32_t* d_cols, double* d_vals, double* d_grad, void* stream);

/* Affine bodies (12 DoF each: translation, then the three 3-vectors of the
 * affine matrix), block rows block_offset + 4 b .. + 3: host mass matrices
 * [n_bodies*144] (row-major 12x12), orthogonality stiffness kappa and volume
 * per body; 16 triplets per body (the lower blocks written as zero blocks,
 * as the affine-body subsystem writes them, abd_linear_subsystem.cu:21-31),
 * Hessian M + the PSD orthogonality Hessian x V dt^2
 * (affine_body/constitutions/ortho_potential.cu:37-70), gradient
 * M (q - q_tilde) + the orthogonality gradient. */
typedef struct b2gen_abd b2gen_abd;
int b2gen_abd_create(int device, int32_t n_bodies, const double* mass12, const double* kappa,
                     const double* volume, double dt, b2gen_abd** out);
int b2gen_abd_destroy(b2gen_abd* a);
int b2gen_abd_system(b2gen_abd* a, const double* d_q, const double* d_qtilde, int32_t block_offset,
                     int32_t* d_rows, int32_t* d_cols, double* d_vals, double* d_grad, void* stream);
/* IPC normal contact of point-triangle (p, t0, t1, t2) and edge-edge
 * (a0, a1, b0, b1) pairs (host lists in global block rows, is_ee per pair,
 * mollifier thresholds eps = 1e-3 |ea_rest|^2 |eb_rest|^2 per pair), barrier
 * kappa dt^2 B(D) with activation distance dhat: the pair's closest-feature
 * type, the exact Hessian projected to PSD for point-triangle / edge-edge
 * types and mollified pairs, the closed rank-1 form for point-edge /
 * point-point types, as the reference's default contact model
 * (contact_system/contact_models/ipc_simplex_normal_contact.cu:320-680).
 * 10 triplets per pair from slot 0 of the given arrays; each pair's gradient
 * is ADDED to d_grad (which holds the other producers' sums), per vertex in
 * pair order. */
typedef struct b2gen_contacts b2gen_contacts;
int b2gen_contacts_create(int device, int32_t n_pairs, const int32_t* pairs, const uint8_t* is_ee,
                          const double* eps, double dhat, double kappa, double dt, b2gen_contacts** out);
int b2gen_contacts_destroy(b2gen_contacts* c);
/* closest-feature type of every pair at the last b2gen_contacts_system
 * (0 point-point, 1 point-edge, 2 point-triangle, 3 edge-edge, -1 beyond dhat) */
int b2gen_contacts_types(b2gen_contacts* c, int8_t* h_types);
int b2gen_contacts_system(b2gen_contacts* c, const double* d_x, int32_t* d_rows, int32_t* d_cols,
                          double* d_vals, double* d_grad, void* stream);
/* The line search's contact term at device state d_x: the sum over the
 * pairs of kappa dt^2 B(D) (times the edge-edge mollifier below eps), the
 * energy b2gen_contacts_system differentiates, in a fixed order (the
 * barrier energy of contact_system/contact_models/ipc_simplex_normal_contact.cu
 * that the line search's compute_energy adds, engine/advance_ipc.cu:515-540). */
int b2gen_contacts_energy(b2gen_contacts* c, const double* d_x, double* h_energy, void* stream);
/* The trajectory filter's step bound over the pairs for the move
 * alpha * d_dx from d_x (the simplex trajectory filter's filter_toi,
 * collision_detection/filters/lbvh_simplex_trajectory_filter.cu:876-1010 with
 * utils/distance/details/ccd.inl, reduced as
 * global_trajectory_filter.cu:111-134): per pair a swept-AABB test expanded
 * by dhat, then additive CCD (eta 0.1, thickness 0, at most 1000 advances);
 * *h_toi = min(1, the smallest time of impact), as a fraction of the move.
 * The candidate pairs are the caller's (no BVH broad phase here). */
int b2gen_contacts_toi(b2gen_contacts* c, const double* d_x, const double* d_dx, double alpha, double* h_toi,
                       void* stream);
/* Candidate detection of the line search's trajectory filter: the
 * point-triangle (surface vertex, surface triangle) and edge-edge (surface
 * edge pairs) candidates whose swept boxes over the move alpha * d_dx come
 * within dhat (the far test of utils/distance/details/ccd.inl:
 * point_triangle_ccd_broadphase / edge_edge_ccd_broadphase), pairs sharing a
 * vertex excluded -- what the simplex trajectory filter collects with its BVH
 * (collision_detection/filters/lbvh_simplex_trajectory_filter.cu:1100-1300).
 * Here a uniform grid of the given cell size (about one surface edge length)
 * hashed into buckets; the pairs come out in a fixed order (point-triangle by
 * vertex, then edge-edge by edge, each by cell and primitive id), in the
 * b2gen_contacts_create layout (p, t0, t1, t2) / (a0, a1, b0, b1).
 * b2gen_trajectory_toi runs the detection and then the narrow phase of
 * b2gen_contacts_toi over the candidates: min(1, the smallest time of impact).
 * A swept box that spans more than 64 cells on an axis (a primitive or a move
 * far larger than the cell) or is not finite makes the call fail with
 * B2S_ERR_ARGUMENT: choose the cell from the largest primitives of the surface.
 * Vertex ids index the state vectors (3 doubles per vertex). */
typedef struct b2gen_trajectory b2gen_trajectory;
int b2gen_trajectory_create(int device, int32_t n_verts, int32_t n_surf_verts, const int32_t* surf_verts,
                            int32_t n_surf_edges, const int32_t* surf_edges, int32_t n_surf_tris,
                            const int32_t* surf_tris, double dhat, double cell, b2gen_trajectory** out);
int b2gen_trajectory_destroy(b2gen_trajectory* t);
/* h_counts[2]: point-triangle and edge-edge candidates found */
int b2gen_trajectory_detect(b2gen_trajectory* t, const double* d_x, const double* d_dx, double alpha,
                            int64_t* h_counts, void* stream);
/* the last detection's candidates: h_pairs[4 * n], h_is_ee[n], n = the two counts summed */
int b2gen_trajectory_pairs(b2gen_trajectory* t, int32_t* h_pairs, uint8_t* h_is_ee);
int b2gen_trajectory_toi(b2gen_trajectory* t, const double* d_x, const double* d_dx, double alpha, double* h_toi,
                         void* stream);
const char* b2gen_trajectory_last_error(void);
const char* b2gen_shell_last_error(void);

#ifdef __cplusplus
}
#endif
