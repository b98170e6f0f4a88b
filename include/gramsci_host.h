/*
 * gramsci_host.h -- host-side pieces of the `gramsci` command-line driver
 * (libgramsci_host.so): option parsing, catalogue reading, weight
 * normalisation and the output writers of the reference program.  They need
 * no GPU and are exported so that they can be tested on their own.
 *
 * The reference keeps these inside its main program (csabiu/Gramsci,
 * src/gramsci.F90); each function cites the lines it replaces.
 */
#ifndef GRAMSCI_HOST_H
#define GRAMSCI_HOST_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parsed command line, the reference's option variables
 * (default_params, src/gramsci.F90:1627-1652; parseOptions :1166-1273). */
typedef struct grh_options {
  char gal[2048];
  char ran[2048];
  char out[2048];
  char cut[2048];
  double rmin, rmax;
  int32_t nbins, nmu;
  int32_t rsd, logbins, cut_mode, mpi, rancat;
  int32_t two_pcf, three_pcf, four_pcf, equi, tetra;
  int32_t gcol;           /* -gcol: region files carry the gal column */
  int32_t help;           /* -help given, or fewer than 6 arguments */
  int32_t error;          /* 0 ok, 1 unknown option, 2 unreadable value */
  char message[256];
} grh_options;

/* Parse argv (argv[0] is the program).  Options are matched on their first
 * six characters, as the reference's character(len=6) option buffer does. */
int grh_parse_args(int argc, const char* const* argv, grh_options* out);

/* Catalogue reading (count_files_2 + read_files_2, src/gramsci.F90:1319-1391):
 * list-directed reads of x y z w per record, galaxies then randoms.
 * Returns the number of points in *n_data / *n_rand; xyz (3N, interleaved)
 * and w (N) are malloc'ed and must be released with grh_free. */
int grh_read_catalogue(const char* gal, const char* ran, double** xyz, double** w,
                       int64_t* n_data, int64_t* n_rand);
/* Region file of -cut mode (count_files + read_files, :1304-1362): records
 * x y z w buffer; all points are data and weights are not normalised. */
int grh_read_region(const char* path, double** xyz, double** w, int32_t** buffer, int64_t* n);
/* -gcol variant (not in the reference): records x y z w gal buffer, the
 * files gramsci-decompose writes.  gal != 0 marks a galaxy; galaxies are
 * returned first, then randoms, each in file order; weights as written. */
int grh_read_region_gal(const char* path, double** xyz, double** w, int32_t** buffer,
                        int64_t* n_data, int64_t* n_rand);
void grh_free(void* p);

/* Region files (domain_decomposition, src/domain_decomposition.f90:1-84).
 *
 * allpoints != NULL: the reference program.  Records x y z w gal aux region
 * read as single precision; region j = 1..max(region) gets the bounding box
 * of its points, the box grown by rmax (single precision), and every point
 * strictly inside the grown box is written to <prefix>j.loadnodes as
 * x y z w gal buffer, buffer = 0 inside the region's own box.
 *
 * allpoints == NULL: the same files from the catalogues gal (+ ran), with
 * region labels from nsplit^3 equal subcubes of the catalogue's bounding
 * box, FP64 throughout (values written with 17 digits), weights normalised
 * over the whole catalogue (galaxies w/sum, randoms -w/sum) and gal = 1 for
 * galaxies, 0 for randoms.  Running `gramsci -cut j.loadnodes -gcol` on each
 * file and summing the tables (grh_resum) gives the unsplit run's table.
 *
 * *nregion receives the number of region files written.  Returns 0, or -1
 * for an unreadable input, -2 for an unwritable output, -3 for bad args. */
int grh_decompose(const char* allpoints, const char* gal, const char* ran, double rmax,
                  int32_t nsplit, const char* prefix, int32_t* nregion);

/* Sum of region tables (the reference's missing resum step): N2 and N3 are
 * summed, N2/N3 recomputed; the bin columns must agree.  query: 2 (2PCF),
 * 3 (3PCF), 4 (4PCF), 5 (-equi), 6 (-tetra).  The disconnected 4PCF/-tetra
 * columns are ratios of sums that a table does not hold; they are written
 * as NaN.  Returns 0, -1 unreadable input, -2 unwritable output, -3
 * mismatched tables. */
int grh_resum(int32_t query, int32_t n, const char* const* inputs, const char* out);

/* Weight normalisation (:1390-1391), sums left to right. */
void grh_normalise(double* w, int64_t n_data, int64_t n_rand);

/* radial_bins(1..nbins+1) (:88-96). */
void grh_radial_bins(double rmin, double rmax, int32_t nbins, int32_t logbins, double* edges);

/* Fortran E14.7 edit descriptor, as gfortran writes it: 14 characters plus
 * a terminating NUL. */
void grh_format_e14_7(double v, char* out15);

/* Output files (:382-397, :513-543, :829-858).  Arrays in the library's
 * layouts (gramsci_cuda.h).  Return 0 on success. */
int grh_write_2pcf(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3);
int grh_write_3pcf(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3);
int grh_write_4pcf(const char* path, const double* edges, int32_t nbins, const double* N2,
                   const double* N3, const double* discN, const double* discR);
/* -equi (:451-459) and -tetra (:648-660) tables; no header line. */
int grh_write_equi(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                   const double* N2, const double* N3);
int grh_write_tetra(const char* path, const double* edges, int32_t nbins, int32_t nmu,
                    const double* N2, const double* N3, const double* discN, const double* discR);

#ifdef __cplusplus
}
#endif

#endif /* GRAMSCI_HOST_H */
