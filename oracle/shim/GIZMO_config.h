/* Compile-time configuration of the reference build used as the CPU oracle:
 * tree-only self-gravity, non-periodic, no hydro modules, OpenMP threads,
 * potential evaluated during the force walk. */
#define IO_DISABLE_HDF5
#define OPENMP 2
#define EVALPOTENTIAL
#define INPUT_IN_DOUBLEPRECISION
