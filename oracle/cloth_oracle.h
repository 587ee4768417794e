/*
 * cloth_oracle.h — C entry points of the CPU oracle (a restatement of the
 * SolidCloth per-substep PBD step, see cloth_oracle.cpp).
 *
 * TEST INFRASTRUCTURE ONLY: called by tests/ as the checker and by bench.py's
 * cpu_baseline leg; never by the shipped library.
 *
 * The entry points deliberately mirror oracle/refbuild/ref_harness.cpp so the
 * same Python driver runs the reference build (oracle/_ref) and this port.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

void* orc_create(void);
void orc_destroy(void* h);
void orc_add_walls(void* h, const float* box6);
void orc_add_sphere(void* h, float cx, float cy, float cz, float r);
void orc_add_sdf(void* h, int nx, int ny, int nz, const float* box6, const float* values);
void orc_add_mesh(void* h, int nv, const float* verts, int nt, const unsigned* idx);
void orc_init_grid(void* h, int divX, int divY, float inc, float ox, float oy, float oz, int horizontal, int attached);
void orc_set_params(void* h, const float* p, int n);
void orc_set_ccd(void* h, int on);
/* ClothModel::SetSolver: 0 Jacobi, 1 Gauss-Seidel (default), 2.. conjugate residual */
void orc_set_solver(void* h, int type);
int orc_num_particles(void* h);
int orc_num_tris(void* h);
int orc_num_bends(void* h);
int orc_num_edges(void* h);
void orc_set_positions(void* h, const float* pos);
void orc_set_state(void* h, const float* pos, const float* prev, const float* vel);
void orc_set_masses(void* h, const float* masses);
void orc_set_inv_mass(void* h, int i, float w);
void orc_get_state(void* h, float* pos, float* prev, float* vel, float* invMass);
float orc_residual(void* h);
void orc_get_tris(void* h, unsigned* idx, float* rest10);
void orc_get_bends(void* h, unsigned* idx);
void orc_get_edges(void* h, int* e4);
/* Check mode: solve FEM triangles / bends in this order (permutations of
   0..T-1 / 0..B-1); NULL restores index order. */
void orc_set_tri_order(void* h, const int* order, int n);
void orc_set_bend_order(void* h, const int* order, int n);
/* Check mode for multi-vertex contacts: 0 = list order (reference), 1 = the
   GPU's deterministic independent-set colouring order (colour, then list index). */
void orc_set_contact_order(void* h, int mode);
void orc_set_link_order(void* h, const int* order, int n);
/* static colours of the triangles and collision-mesh edges (and their counts):
   the GPU's order of triangle / edge collider contacts in check mode */
void orc_set_static_colours(void* h, const int* triColour, int nt, int nTriColours, const int* edgeColour, int ne,
                            int nEdgeColours);
void orc_load_topology(void* h, int n, const float* pos, const float* invMass, int nt, const unsigned* tri,
                       const float* rest10, int nb, const unsigned* bend4, int nl, const unsigned* link2,
                       const float* linkRest2);
int orc_num_links(void* h);
void orc_get_links(void* h, unsigned* idx2, float* lenStiff);
void orc_set_portable_math(int on);
float orc_portable_acos(float x);
void orc_step(void* h, float dt);
void orc_update_mesh(void* h);
void orc_predict_detect(void* h, float hh, int runCCD);
int orc_num_contacts(void* h, int kind);
void orc_get_vertex_contacts(void* h, int* idx2, float* f7);
void orc_get_tri_contacts(void* h, int* idx4, float* f9);
void orc_get_edge_contacts(void* h, int* idx3, float* f8);
void orc_get_self_contacts(void* h, int kind, int* idx4, float* f7);
void orc_get_mesh_normals(void* h, int prev, float* n);
void orc_get_mesh_tri_normals(void* h, int prev, float* n);
/* colour of each self contact under the independent-set colouring (kind 3/4) */
void orc_self_contact_colours(void* h, int kind, int* colours);
/* Continuous self-collision: all-pairs swept-box broad phase and narrow phase.
   The broad phase sweeps boxes sorted by min x (exact: the all-pairs set);
   orc_set_bruteforce_broadphase(h, 1) selects the plain all-pairs loop. */
void orc_set_bruteforce_broadphase(void* h, int on);
int orc_ccd_broadphase(void* h, float tol, int kind, int* pairs, int cap);
void orc_ccd_narrow_on(void* h, int nvt, const int* vt, int nee, const int* ee);
void orc_swept_boxes(void* h, int kind, float tol, float* out);

#ifdef __cplusplus
}
#endif
