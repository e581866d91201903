// Synthetic Newton-system generator for the linear-solve workloads.
//
// Produces the raw input of one Newton-step linear solve exactly in the
// conventions libuipc's CUDA backend hands to GlobalLinearSystem:
//   * raw 3x3 Hessian triplets (row, col, value) with row <= col in the global
//     block numbering (producers write only the block-upper half, transposing a
//     block when its local order is reversed; see
//     src/backends/cuda/finite_element/constitutions/stable_neo_hookean_3d.cu:252-263
//     in libuipc),
//   * values as Eigen::Matrix3d would store them (9 doubles, column-major),
//   * duplicates NOT summed (one block per element stencil entry),
//   * the gradient b of E = 1/2|x - x_tilde|_M^2 + dt^2 * (Psi + barrier),
//     so that the solve is A x = b and the Newton direction is dx = -x
//     (src/backends/cuda/finite_element/fem_linear_subsystem.cu:119-126).
//
// This is input synthesis for tests and benchmarks; it is host C++ only.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b2g_config
{
    int    scene;          // 1 = cubes stacked along +y on a ground plane, 2 = twisted bar,
                           // 3 = cloth over affine bodies, 4 = cube grid + cloth + bodies
    int    cells_x;        // cells per cube edge (x)
    int    cells_y;        // (y)
    int    cells_z;        // (z)
    int    n_cubes;        // cubes stacked along +y (scene 1)
    double h;              // cell edge length [m]
    double jitter;         // vertex jitter amplitude as a fraction of h (uniform +-)
    double normal_jitter;  // contact-face normal jitter amplitude [m] (scene 1, n_cubes > 1)
    double gap;            // nominal gap between stacked cubes [m]
    uint64_t seed;
    double E;              // Young's modulus [Pa]
    double nu;             // Poisson ratio
    double rho;            // density [kg/m^3]
    double dt;             // time step [s]
    double gravity;        // gravity along -y [m/s^2]
    double dhat;           // barrier activation distance [m]
    double kappa;          // barrier stiffness [Pa]
    double ground_offset;  // ground plane sits this far below the lowest vertex [m]
    double twist_deg;      // scene 2: end rotation (+-) about the bar axis [deg]
    int    n_threads;      // OpenMP threads (0 = default)
    // scene 3 (cloth draped over affine bodies): cells_x = cloth vertices per
    // side, n_cubes = bodies per side, E = cloth stretch stiffness [N/m]
    double body_kappa;     // affine-body orthogonality stiffness [Pa]
    double bend_k;         // cloth bending stiffness [N m]
    double cloth_size;     // cloth side length [m]
    // scene 4 (cube grid + cloth + bodies): n_cubes = cubes per grid side,
    // cells_x/y/z = cells per cube edge, E / nu / rho the cubes' material
    double wall_gap;       // gap between neighbouring cubes of the grid [m]
    int    cloth_n;        // cloth vertices per side
    int    bodies_x;       // affine bodies along x
    int    bodies_z;       // affine bodies along z
    double cloth_k;        // cloth stretch stiffness [N/m] (scene 4)
} b2g_config;

typedef struct b2g_system b2g_system;

// Fill `cfg` with the defaults of the 10x10x10 cube-on-ground case.
void b2g_default_config(b2g_config* cfg);

// Generate one Newton system. Returns 0 on success, non-zero on error
// (message through b2g_last_error()).
int b2g_generate(const b2g_config* cfg, b2g_system** out);
// The Newton system of the same mesh at a given state: x = current positions,
// x_tilde = x_prev + dt v + dt^2 g (both [n_verts*3]). The ground plane stays
// where the rest shape puts it; in the twisted bar the end layers are fixed
// (the caller places them). Used to step a scene through time.
int b2g_generate_state(const b2g_config* cfg, const double* x, const double* x_tilde, b2g_system** out);
void b2g_free(b2g_system* sys);
const char* b2g_last_error(void);

// Sizes
int64_t b2g_num_verts(const b2g_system* s);
int64_t b2g_num_tets(const b2g_system* s);
int64_t b2g_num_triplets(const b2g_system* s);
int64_t b2g_num_contacts(const b2g_system* s);  // PT + EE + ground pairs (scene 3: cloth-body pairs)
// scene 3: affine bodies come first in the DoF order, 4 block rows (12 DoF:
// translation, then the 3 columns of the affine matrix) per body; the cloth
// vertices follow from block row 4 * n_bodies on
int64_t b2g_num_bodies(const b2g_system* s);

// Data (owned by the system; valid until b2g_free)
const double* b2g_positions(const b2g_system* s);    // [n_verts*3]
const double* b2g_rest_positions(const b2g_system* s);  // [n_verts*3]
const int32_t* b2g_tets(const b2g_system* s);         // [n_tets*4]
const int32_t* b2g_triplet_rows(const b2g_system* s); // [n_triplets]
const int32_t* b2g_triplet_cols(const b2g_system* s); // [n_triplets]
const double*  b2g_triplet_vals(const b2g_system* s); // [n_triplets*9] column-major 3x3
const double*  b2g_gradient(const b2g_system* s);     // [n_verts*3]

// Vertex adjacency from tetrahedra (sorted, unique, CSR) -- the MAS
// neighbour graph built by FEMMASPreconditioner::do_init
// (src/backends/cuda/finite_element/fem_mas_preconditioner.cu:157-200).
int64_t        b2g_num_adjacency(const b2g_system* s);
const int32_t* b2g_adjacency_start(const b2g_system* s);  // [n_verts+1]
const int32_t* b2g_adjacency_list(const b2g_system* s);   // [num_adjacency]

// Element routines of the cloth / affine-body energies (elements.h), for
// checks against the formulas: energy, gradient and Hessian (row-major) of
//  * one Baraff-Witkin triangle: x[9] current and rest[9] rest corners,
//    weight w (the element scale; the energy is returned unscaled);
//  * one discrete-shell hinge (x0, x1, x2, x3; edge x1-x2) with its rest
//    corners, stiffness kappa, weight w (Gauss-Newton Hessian);
//  * the orthogonality potential of q[12] (gradient/Hessian over q[3..11],
//    Hessian projected to PSD), weight w.
double b2g_element_bw(const double* x, const double* rest, double stretch, double shear, double rate, double w,
                      double* G9, double* H81);
double b2g_element_dsb(const double* x, const double* rest, double kappa, double w, double* G12, double* H144);
double b2g_element_ortho(const double* q, double kappa, double w, double* G9, double* H81);
// one contact pair X[12] ((p, t0, t1, t2) or, with is_ee, (a0, a1, b0, b1)),
// mollifier threshold eps, dhat, k = kappa dt^2: gradient and Hessian over the
// 4 vertices; returns the closest-feature type (0 PP, 1 PE, 2 PT, 3 EE) or -1
// beyond dhat
int b2g_element_contact(const double* X, int is_ee, double eps, double dhat, double k, double* G12, double* H144);
// the pair's barrier energy (the energy b2g_element_contact differentiates)
double b2g_contact_energy(const double* X, int is_ee, double eps, double dhat, double k);
// additive CCD of the pair moving by dX[12] over the step (eta, thickness xi,
// at most max_iter advances, no hit past toi_max): 1 and *toi on a hit, else 0
// (*toi = toi_max)
int b2g_accd(const double* X, const double* dX, int is_ee, double eta, double xi, int max_iter, double toi_max,
             double* toi);

#ifdef __cplusplus
}
#endif
