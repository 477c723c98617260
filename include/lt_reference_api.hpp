/*
 * lt_reference_api.hpp -- the reference's C++ host entry points of the lensing-map path,
 * with their exact signatures (type_t = double), implemented on top of liblt_b200.so.
 *
 * A caller built against Lenstool-HPC's headers links against liblt_b200.so instead of
 * liblenstoolhpc_GPU.so and keeps its calls unchanged.  The struct types below repeat
 * the member lists of the reference's src/structure_hpc.hpp (same order and types, so
 * the layouts match); only the types these functions take are declared.
 *
 * Semantics kept: host pointers in the *_GPU wrappers (synchronous), device pointers in
 * the *_CPU_GPU launchers (asynchronous on the legacy stream), square-grid overloads that
 * derive dx, dy from the frame.  Differences: no process exit on errors (a message is
 * printed and the outputs are left untouched), any grid shape, no sentinel read.
 */
#ifndef LT_REFERENCE_API_HPP
#define LT_REFERENCE_API_HPP

#include <string>

#ifndef LT_REFERENCE_TYPES_DEFINED
#define LT_REFERENCE_TYPES_DEFINED
typedef double type_t;

/* src/structure_hpc.hpp:84-141 */
struct point { type_t x, y; };
struct matrix { type_t a, b, c, d; };

/* src/structure_hpc.hpp:445-454 */
struct grid_param { type_t xmin, xmax, ymin, ymax, lmin, lmax, rmax; };

/* src/structure_hpc.hpp:468-478 */
struct cosmo_param {
    int model;
    type_t omegaM, omegaX, curvature, wX, wa, H0, h;
};

/* src/structure_hpc.hpp:257-287 (field pointers; type is sorted into runs) */
struct Potential_SOA {
    int *type;
    char type_name[10];
    type_t *name;
    type_t *position_x, *position_y;
    type_t *weight, *b0, *vdisp;
    type_t *ellipticity_angle, *ellipticity, *ellipticity_potential;
    type_t *rcore, *rcut, *rscale, *exponent, *alpha, *einasto_kappacritic;
    type_t *z, *mag, *lum, *theta;
    type_t *anglecos, *anglesin;
    type_t *sigma, *dlsds;
    int *SOA_index;
    int *N_types;
};

/* src/structure_hpc.hpp:354-424 (N_MAX_POTFILE = 10, NTYPES = 2) */
struct runmode_param {
    int nbgridcells;
    int source;
    int nsets;
    int image;
    int N_z_param;
    int nimagestot;
    int multi;
    type_t ref_ra, ref_dec;
    int mass, mass_gridcells;
    type_t z_mass, z_mass_s;
    std::string mass_name;
    int potential, pot_gridcells;
    type_t z_pot;
    std::string pot_name;
    int nhalos, n_tot_halos;
    int potfile;
    int npotfile[10];
    int Nb_potfile;
    int dpl, dpl_gridcells;
    type_t z_dpl;
    std::string dpl_name1, dpl_name2;
    int inverse, arclet, debug;
    int grid, gridcells;
    type_t zgrid;
    int cline;
    int amplif, amplif_gridcells;
    type_t z_amplif;
    std::string amplif_name;
    int shear, shear_gridcells;
    type_t z_shear;
    std::string shear_name;
    int time;
    int Nlens[2];
    std::string imagefile;
    std::string potfilename[10];
    std::string sourfile;
};
#endif

/* map epilogue function types: src/grid_map_ampli_GPU.cuh:35-38, src/grid_map_pot_GPU.cuh:35-38 */
typedef void (*map_gpu_function_t)(type_t *map, type_t *grid_grad2_a, type_t *grid_grad2_b, type_t *grid_grad2_c,
                                   type_t *grid_grad2_d, type_t dl0s, type_t dos, type_t dl, type_t h, type_t z,
                                   int nbgridcells_x, int nbgridcells_y, const struct grid_param *frame);
typedef void (*map_pot_function_t)(type_t *map, type_t dl0s, type_t dos, type_t dl, type_t h, type_t z,
                                   int nbgridcells_x, int nbgridcells_y, const struct grid_param *frame);

/* deflection: src/grid_gradient_GPU.cuh:34-41 */
void gradient_grid_GPU(type_t *grid_grad_x, type_t *grid_grad_y, const struct grid_param *frame,
                       const struct Potential_SOA *lens, int nhalos, int nbgridcells);
void gradient_grid_GPU(type_t *grid_grad_x, type_t *grid_grad_y, const struct grid_param *frame,
                       const struct Potential_SOA *lens, int nhalos, type_t dx, type_t dy, int nbgridcells_x,
                       int nbgridcells_y, int istart = 0, int jstart = 0);
void gradient_grid_GPU_UM(type_t *grid_grad_x, type_t *grid_grad_y, const struct grid_param *frame,
                          const struct Potential_SOA *lens, int nhalos, type_t dx, type_t dy, int nbgridcells_x,
                          int nbgridcells_y, int istart, int jstart);
void module_potentialDerivatives_totalGradient_SOA_CPU_GPU(type_t *grid_grad_x, type_t *grid_grad_y,
                                                           const struct grid_param *frame,
                                                           const struct Potential_SOA *lens_gpu, int nbgridcells,
                                                           int nhalos);
void module_potentialDerivatives_totalGradient_SOA_CPU_GPU(type_t *grid_grad_x, type_t *grid_grad_y,
                                                           const struct grid_param *frame,
                                                           const struct Potential_SOA *lens, int nhalos, type_t dx,
                                                           type_t dy, int nbgridcells_x, int nbgridcells_y,
                                                           int istart, int jstart);

/* Hessian: src/grid_gradient2_GPU.cuh:32-43 */
void gradient2_grid_GPU(type_t *grid_grad2_a, type_t *grid_grad2_b, type_t *grid_grad2_c, type_t *grid_grad2_d,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int nbgridcells);
void gradient2_grid_GPU(type_t *grid_grad2_a, type_t *grid_grad2_b, type_t *grid_grad2_c, type_t *grid_grad2_d,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int nhalos, type_t dx,
                        type_t dy, int nbgridcells_x, int nbgridcells_y, int istart = 0, int jstart = 0);
void module_potentialDerivatives_totalGradient2_SOA_CPU_GPU(type_t *grid_grad2_a, type_t *grid_grad2_b,
                                                            type_t *grid_grad2_c, type_t *grid_grad2_d,
                                                            const struct grid_param *frame,
                                                            const struct Potential_SOA *lens_gpu, int nbgridcells,
                                                            int nhalos);
void module_potentialDerivatives_totalGradient2_SOA_CPU_GPU(type_t *grid_grad2_a, type_t *grid_grad_b,
                                                            type_t *grid_grad2_c, type_t *grid_grad_d,
                                                            const struct grid_param *frame,
                                                            const struct Potential_SOA *lens, int nhalos, type_t dx,
                                                            type_t dy, int nbgridcells_x, int nbgridcells_y,
                                                            int istart, int jstart);
void module_potentialDerivatives_Kmap_SOA_CPU_GPU(type_t *grid_grad2_a, type_t *grid_grad2_b, type_t *grid_grad2_c,
                                                  type_t *grid_grad2_d, const struct grid_param *frame,
                                                  const struct Potential_SOA *lens_gpu, int nhalos, type_t dx,
                                                  type_t dy, int nbgridcells_x, int nbgridcells_y, int istart,
                                                  int jstart);

/* potential: src/grid_potential_GPU.cuh:31-32 */
void potential_grid_GPU(type_t *potential, const struct grid_param *frame, const struct Potential_SOA *lens,
                        int nhalos, int nbgridcells);
void module_potential_SOA_CPU_GPU(type_t *potential, const struct grid_param *frame, const struct Potential_SOA *lens,
                                  int nhalos, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y, int istart,
                                  int jstart);

/* maps: src/grid_map_{ampli,shear,mass,pot,dpl}_GPU.cuh */
map_gpu_function_t select_map_ampli_function(const struct runmode_param *runmode);
map_gpu_function_t select_map_shear_function(const struct runmode_param *runmode);
map_gpu_function_t select_map_mass_function(const struct runmode_param *runmode);
map_pot_function_t select_map_potential_function(const struct runmode_param *runmode);

void map_grid_ampli_GPU(map_gpu_function_t mapfunction, type_t *amplif, const struct cosmo_param *cosmo,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int nbgridcells,
                        int mode_amp, type_t z);
void map_grid_ampli_GPU(map_gpu_function_t mapfunction, type_t *amplif, const struct cosmo_param *cosmo,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int mode_amp,
                        type_t z, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y, int istart = 0,
                        int jstart = 0);
void map_grid_shear_GPU(map_gpu_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int nbgridcells,
                        int mode_amp, type_t z);
void map_grid_shear_GPU(map_gpu_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                        const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int mode_amp,
                        type_t z, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y, int istart = 0,
                        int jstart = 0);
void map_grid_mass_GPU(map_gpu_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                       const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int nbgridcells,
                       int mode_amp, type_t zl, type_t zs);
void map_grid_mass_GPU(map_gpu_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                       const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int mode_amp,
                       type_t zl, type_t zs, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y,
                       int istart = 0, int jstart = 0);
void map_grid_potential_GPU(map_pot_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                            const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens,
                            int nbgridcells, int mode_amp, type_t z);
void map_grid_potential_GPU(map_pot_function_t mapfunction, type_t *map, const struct cosmo_param *cosmo,
                            const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int mode_amp,
                            type_t z, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y, int istart = 0,
                            int jstart = 0);
void map_grid_dpl_GPU(map_gpu_function_t mapfunction, type_t *dplx, type_t *dply, const struct cosmo_param *cosmo,
                      const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int nbgridcells,
                      int mode_amp, type_t z);
void map_grid_dpl_GPU(map_gpu_function_t mapfunction, type_t *dplx, type_t *dply, const struct cosmo_param *cosmo,
                      const struct grid_param *frame, const struct Potential_SOA *lens, int Nlens, int mode_amp,
                      type_t z, type_t dx, type_t dy, int nbgridcells_x, int nbgridcells_y, int istart = 0,
                      int jstart = 0);

/* map epilogues on device Hessian planes (the functions select_map_*_function returns):
 * src/grid_map_ampli_GPU.cu:306-547, src/grid_map_shear_GPU.cu:187-369,
 * src/grid_map_mass_GPU.cu:219-322, src/grid_map_pot_GPU.cu:180-273 */
#define LT_MAP_FN(name)                                                                                            \
    void name(type_t *map, type_t *a, type_t *b, type_t *c, type_t *d, type_t dl0s, type_t ds, type_t dl, type_t h, \
              type_t z, int nx, int ny, const struct grid_param *frame)
LT_MAP_FN(amplif_1_grid_CPU_GPU);
LT_MAP_FN(amplif_2_grid_CPU_GPU);
LT_MAP_FN(amplif_3_grid_CPU_GPU);
LT_MAP_FN(amplif_4_grid_CPU_GPU);
LT_MAP_FN(amplif_5_grid_CPU_GPU);
LT_MAP_FN(amplif_6_grid_CPU_GPU);
LT_MAP_FN(shear_1_grid_CPU_GPU);
LT_MAP_FN(shear_2_grid_CPU_GPU);
LT_MAP_FN(shear_3_grid_CPU_GPU);
LT_MAP_FN(shear_4_grid_CPU_GPU);
LT_MAP_FN(mass_1_grid_CPU_GPU);
LT_MAP_FN(mass_2_grid_CPU_GPU);
LT_MAP_FN(mass_3_grid_CPU_GPU);
LT_MAP_FN(mass_4_grid_CPU_GPU);
#undef LT_MAP_FN
void potential_1_grid_CPU_GPU(type_t *potential, type_t dl0s, type_t ds, type_t dl, type_t h, type_t z, int nx,
                              int ny, const struct grid_param *frame);
void potential_2_grid_CPU_GPU(type_t *potential, type_t dl0s, type_t ds, type_t dl, type_t h, type_t z, int nx,
                              int ny, const struct grid_param *frame);
void dpl_grid_CPU_GPU(type_t *map, type_t dl0s, type_t ds, type_t dl, type_t h, type_t z, int nx, int ny,
                      const struct grid_param *frame);

/* reference-API errors are reported here (the reference exits instead) */
extern "C" int lt_reference_api_last_status(void);

#endif /* LT_REFERENCE_API_HPP */
