/* Compile-time configuration of the reference build used as the CPU oracle:
 * tree-only self-gravity, non-periodic, no hydro modules, OpenMP threads,
 * potential evaluated by compute_potential after the force walk (the
 * build variant that pins the potential-only walk). */
#define IO_DISABLE_HDF5
#define OPENMP 2
#define COMPUTE_POTENTIAL_ENERGY
#define INPUT_IN_DOUBLEPRECISION
