/*
 * cosims_host.h -- C ABI of the host side: input-file parameters, molecule
 * import and the per-molecule setup that the trajectory path consumes.
 *
 * Replaces the reference's setup chain (main.cpp:106-138):
 *   fileParams::interpretCMD / setDefaultParams / importParams
 *     (fileParams.cpp:78-510) -> cosims_config_defaults / cosims_config_read
 *   molecule2::importMFJ / importPDB / importFile / setMolProperties /
 *     printMolStats (molecule2.cpp:132-938, 1131-1391)
 *   monteTraj::monteTraj (monteTraj.cpp:26-142): velocity distribution,
 *     impactParam::setBoundry / findEllipsoidBound / printBoundryResults
 *     (impactParam.cpp:602-1056), forceAccel::setClusters + PCM_Cluster
 *     (forceAccel.cpp:53-210, PCM_Cluster.cpp:38-249)
 *                                   -> cosims_setup_create
 * The setup keeps the reference's arithmetic, so the molecule, ellipsoid and
 * clusters it produces are the reference's bit for bit (the trajectory path's
 * parity depends on it).
 */
#ifndef COSIMS_HOST_H
#define COSIMS_HOST_H

#include <stdint.h>
#include "cosims_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Every key of the reference's input file (fileParams.cpp:314-468), its
 * command line (-n -s) and the derived values the rest of the program reads.
 * Field names follow the input-file keys. */
typedef struct cosims_config {
    char name[256];            /* name (default: molecule file stem; "_<charge>"
                                  is appended after an input file is read)     */
    char dir[1024];            /* dir: output directory ("" = working dir)      */
    double dt;                 /* dt (ps)                                        */
    double temp;               /* temp (K)                                       */
    int64_t traj;              /* trajectories per integral (key value * 1000)   */
    int32_t iter;              /* iterations (CCS integrals)                     */
    int32_t threads;           /* threads (host threads for the setup scan)      */
    int64_t seed;              /* seed                                           */
    int32_t seed_set;          /* seed came from -s or the input file            */
    double gmax, gmin;         /* parsed, unused (as in the reference)           */
    int32_t print_mol, proj, print_traj, print_traj_fail, print_data, print_data_fail;
    int32_t dispersion_cutoff;
    double dispersion_radius;  /* 0 = sigma_max * (150 / 0.5)^(1/3)              */
    int32_t multipole;
    double multipole_radius;   /* 0 = 20 Angstrom                                */
    int32_t multipole_order;
    int32_t print_rate;
    int32_t display_progress;
    int32_t max_cluster_size;
    double charge;             /* charge key: total charge (0 = none)            */
    int32_t charged;           /* charge_ext                                     */
    int32_t debugging;         /* a debugging key was given                      */
    uint32_t changed;          /* bit per key set by the input file (COSIMS_KEY_*) */
} cosims_config;

#define COSIMS_KEY_NAME    (1u << 0)
#define COSIMS_KEY_CHARGE  (1u << 1)
#define COSIMS_KEY_PRINT_RATE (1u << 2)
#define COSIMS_KEY_THREADS (1u << 3)
#define COSIMS_KEY_SEED    (1u << 4)

/* fileParams::setDefaultParams (fileParams.cpp:203-259) for a molecule file. */
cosims_status cosims_config_defaults(cosims_config *cfg, const char *mol_path);
/* fileParams::importParams (fileParams.cpp:261-510): defaults, then the
 * file's keys.  Messages the reference prints (bad lines, repeated keys) are
 * written to log (may be NULL). */
cosims_status cosims_config_read(cosims_config *cfg, const char *input_path,
                                 const char *mol_path, char *log, int64_t log_cap);

typedef struct cosims_setup cosims_setup;

/* Scalars of a finished setup, for the log and for checks. */
typedef struct cosims_setup_info {
    int32_t n_atoms, n_clusters, n_boundary, force_type;
    double total_mass, mu, total_charge;
    double center[3];          /* centre of mass before centring                 */
    double radius_gyration;
    double inertia[9];         /* inertia tensor before the rotation             */
    double rotation[9];        /* rotation applied (eigenvectors)                */
    double dipole[3], quadrupole[9];
    double ell_a, ell_b, ell_c;/* after enlargement                              */
    double ell_unc[3];         /* axis uncertainties                             */
    double rmsd, avg_axes, avg_axes_unc, surf_area, surf_area_unc, enlarge;
    double cov[9];             /* axis covariance matrix                         */
    double b_max, g_min, g_max, g_mean, g_mode, pct_used;
    double beta, ccs_const, r_disp, r_mp;
    int32_t centers_replaced;
    double avg_cluster_size, avg_cluster_radius;
    /* wall time (ms) of the setup phases: molecule file, force-field terms and
     * rotation, velocity distribution, boundary scan, ellipsoid fit and
     * enlargement, PCM clusters and multipoles */
    double setup_ms[6];
} cosims_setup_info;

/* The whole per-molecule setup.  atom_path: optional atoms.dat (NULL or "").
 * The molecule file type follows its extension (.pdb or .mfj, any case).
 * log (may be NULL) receives the messages the reference writes while
 * importing. */
cosims_status cosims_setup_create(const cosims_config *cfg, const char *mol_path,
                                  const char *atom_path, char *log, int64_t log_cap,
                                  cosims_setup **out);
/* The same setup with the boundary ray march (impactParam::setBoundry's
 * OpenMP loop, impactParam.cpp:661-721) on `device`: one GPU thread per ray,
 * the same IEEE operation sequence, so the result equals cosims_setup_create's
 * bit for bit.  For serving and batches, where host setup time dominates. */
cosims_status cosims_setup_create_device(const cosims_config *cfg, const char *mol_path,
                                         const char *atom_path, int32_t device, char *log,
                                         int64_t log_cap, cosims_setup **out);
/* Multi-structure molecule files (coordinate sets / conformers), for batches
 * fed from files.  The reference reads one coordinate set per run and warns
 * "Multiple coordinate sets not yet supported" (molecule2.cpp:497-501).
 * MFJ: the header's second line is the number of sets K; the records after
 * the header are read line by line, a line of at least five tokens whose first
 * three are numbers being a record and any other line a separator, and set s
 * is records s*N .. s*N+N-1 (N = the header's atom count).  PDB: each
 * MODEL .. ENDMDL block is a set; a file without MODEL records is one set.
 * cosims_molecule_file_structures returns K (1 for a single-structure file). */
cosims_status cosims_molecule_file_structures(const char *mol_path, int32_t *count);
/* cosims_setup_create (device < 0) or cosims_setup_create_device (device >= 0)
 * for coordinate set `structure` (0-based).  Each set gets the whole setup of
 * its own (rotation, boundary, ellipsoid, clusters), so set s equals the setup
 * of a single-structure file holding only set s, bit for bit.  For a
 * single-structure file, set 0 is read exactly as cosims_setup_create reads it. */
cosims_status cosims_setup_create_structure(const cosims_config *cfg, const char *mol_path,
                                            const char *atom_path, int32_t structure,
                                            int32_t device, char *log, int64_t log_cap,
                                            cosims_setup **out);
/* Views of the setup's molecule and path scalars (valid while the setup
 * lives); feed them to cosims_ctx_create. */
cosims_status cosims_setup_molecule(const cosims_setup *s, cosims_molecule *mol,
                                    cosims_params *par);
cosims_status cosims_setup_get_info(const cosims_setup *s, cosims_setup_info *info);
/* Potential-energy boundary points (impactParam::setBoundry); returns count. */
int64_t cosims_setup_boundary(const cosims_setup *s, double *xyz, int64_t cap);
/* Element symbol of atom i (file order), NUL-terminated. */
const char *cosims_setup_atom_symbol(const cosims_setup *s, int32_t i);
void cosims_setup_destroy(cosims_setup *s);

#ifdef __cplusplus
}
#endif
#endif /* COSIMS_HOST_H */
