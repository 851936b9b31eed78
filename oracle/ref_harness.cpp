/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (never linked into the product).
 *
 * A thin extern "C" harness around the UNMODIFIED CoSIMS reference sources.
 * `oracle/Makefile` compiles this file together with the reference's own
 * src/*.cpp (minus main.cpp) straight from the reference checkout into
 * oracle/_ref/libcosims_ref.so.  Tests and tests/golden/make_golden.py use it
 * to pin the oracle restatement (oracle/cosims_oracle.c) and the product's
 * host setup against what the reference itself computes.
 *
 * It reproduces the reference's program flow:
 *   main.cpp:106-138  interpretCMD -> importPDB/importMFJ -> printInfo ->
 *                     printMolStats -> new monteTraj(mol, shared)
 * and then exposes, per trajectory, diffEqSolver::verletVel
 * (diffEqSolver.cpp:81-211), forceAccel::getReducedVec/getPotential
 * (forceAccel.cpp:887-982) and monteTraj::setUpTraj (monteTraj.cpp:174-278).
 *
 * Private members of the reference classes are read through the standard
 * explicit-instantiation access idiom (no reference header is edited).
 */
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <random>
#include "molecule2.h"
#include "monteTraj.h"
#include "diffEqSolver.h"
#include "forceAccel.h"
#include "impactParam.h"
#include "fileParams.h"
#include "myStructs.h"

/* ---- globals that main.cpp:39-91 defines -------------------------------- */
ofstream fileStream_ext;
string omegaFilePath_ext;
string fileLocaiton_ext;
string molFilePath_ext;
string molFileName_ext;
string atomFilePath_ext;
string dataFilePath_ext;
string xyzFilePath_ext;
string iterFilePath_ext;
string name_ext;
string subDir_ext;
string printMolName_ext;
double temp_ext;
double dt_ext;
double mass_ext;
double mu;
int trajNum_ext;
int iterations_ext;
int numThreads_ext;
long long int seed_ext;
int printRate_ext;
int maxClusterSize_ext;
int multipole_order_ext;
double cutOffRadius_ext;
double gMax_ext;
double gMin_ext;
double totalCharge_ext;
bool displayProg_ext;
double dispersion_radius_ext;
double multipole_radius_ext;
bool multipole_ext;
bool dispersionCutoff_ext;
bool charge_ext;
bool projection_ext;
bool shorten_ext;
bool printTraj_ext;
bool printTrajOnFail_ext;
bool printData_ext;
bool printDataOnFail_ext;
bool printMol_ext;
bool printToColsole_ext = false;

/* ---- access to private members (explicit instantiation idiom) ----------- */
template <typename Tag, typename Tag::type M>
struct Robber { friend typename Tag::type get(Tag) { return M; } };

#define ROB(NAME, CLASS, TYPE, MEMBER)                                  \
    struct NAME { typedef TYPE CLASS::*type; friend type get(NAME); };  \
    template struct Robber<NAME, &CLASS::MEMBER>;

ROB(R_gasAtom, monteTraj, diffEqSolver, gasAtom)
ROB(R_impactB, monteTraj, impactParam, impactB)
ROB(R_const1, monteTraj, double, const1)
ROB(R_const2, monteTraj, double, const2)
ROB(R_maxDist, monteTraj, float, maxDist)
ROB(R_maxVelDistr, monteTraj, double, maxVelDistr)
ROB(R_velDistr, monteTraj, VelocityDistribution, velDistr)
ROB(R_clusterGroups, std::forceAccel, vector<vector<int> >, clusterGroups)
ROB(R_clusterPos, std::forceAccel, vector<vector3D<double> >, clusterPos)
ROB(R_clusterRadius, std::forceAccel, vector<double>, clusterRadius)
ROB(R_centerReplace, std::forceAccel, vector<bool>, centerReplace)
ROB(R_totalCharge, std::forceAccel, vector<double>, totalCharge)
ROB(R_dipole, std::forceAccel, vector<vector<double> >, dipole)
ROB(R_quadPole, std::forceAccel, vector<vector<vector<double> > >, quadPole)
ROB(R_forceType, std::forceAccel, int, forceType)
ROB(R_dipoleScalar, std::forceAccel, double, dipoleScalar)
ROB(R_boundry, impactParam, vector<vector3D<double> >, boundryPoints)
ROB(R_enlarge, impactParam, double, enlargeAmount)

static molecule2 *g_mol = nullptr;
static monteTraj *g_monte = nullptr;
static threadSharedParams g_shared;

static std::forceAccel &force() { return ((*g_monte).*get(R_gasAtom())).forceFunct; }

extern "C" {

/* Runs the reference's setup for one molecule.  argv mirrors the command line
 * `cosims -m mol [-i input] [-a atoms] -s seed` (fileParams.cpp:78-201); every
 * output file is written under workdir.  Returns 0 on success. */
int ref_setup(const char *mol_path, const char *input_path, const char *atom_path,
              const char *workdir, long long seed)
{
    std::vector<std::string> args = {"cosims", "-m", mol_path};
    if (input_path && *input_path) { args.push_back("-i"); args.push_back(input_path); }
    if (atom_path && *atom_path) { args.push_back("-a"); args.push_back(atom_path); }
    args.push_back("-s");
    args.push_back(std::to_string(seed));
    std::vector<char *> argv;
    for (auto &s : args) argv.push_back(const_cast<char *>(s.c_str()));
    argv.push_back(nullptr);

    atomFilePath_ext.clear();
    fileParams files;
    char cwd[4096];
    std::snprintf(cwd, sizeof cwd, "%s", workdir);
    if (!files.interpretCMD((int)args.size(), argv.data(), cwd)) return 1;

    g_mol = new molecule2();
    g_mol->totalMass = 0; g_mol->centerX = 0; g_mol->centerY = 0; g_mol->centerZ = 0;
    g_mol->numAtoms = 0;
    if (files.getMolFileExt().compare("pdb") == 0)
        g_mol->importPDB();
    else
        g_mol->importMFJ(files.getNameChanged(), files.getChargeChanged());
    if (g_mol->numAtoms == 0) return 2;
    files.printInfo();
    g_mol->printMolStats();
    g_monte = new monteTraj(*g_mol, g_shared);
    return 0;
}

int ref_num_atoms(void) { return g_mol->numAtoms; }

/* Atoms after COM centring and the inertia rotation, in file order. */
void ref_get_atoms(double *xyz, double *charge, double *sig6, double *eps24m,
                   double *eps4, double *mass)
{
    for (int i = 0; i < g_mol->numAtoms; i++) {
        const dataList &d = g_mol->data[i];
        xyz[3 * i + 0] = d.coords.X;
        xyz[3 * i + 1] = d.coords.Y;
        xyz[3 * i + 2] = d.coords.Z;
        charge[i] = d.charge;
        sig6[i] = d.sigAvg6;
        eps24m[i] = d.eps24_mass;
        eps4[i] = d.eps4;
        mass[i] = d.mass;
    }
}

/* Scalar setup values, in a fixed order (see REF_SCALARS in the Python side). */
int ref_get_scalars(double *out, int cap)
{
    monteTraj &m = *g_monte;
    impactParam &ip = m.*get(R_impactB());
    std::forceAccel &f = force();
    VelocityDistribution &vd = m.*get(R_velDistr());
    double v[] = {
        mass_ext, g_mol->totalMass, m.beta, m.gMin, m.gMax, m.*get(R_maxVelDistr()),
        vd.normFactor(), ip.a, ip.b, ip.c, m.bMax, (double)(m.*get(R_maxDist())),
        m.*get(R_const1()), m.*get(R_const2()), f.*get(R_dipoleScalar()),
        (double)(f.*get(R_forceType())), dispersion_radius_ext, multipole_radius_ext,
        (double)multipole_order_ext, dt_ext, temp_ext, (double)trajNum_ext,
        (double)iterations_ext, (double)printRate_ext, (double)projection_ext,
        (double)charge_ext, totalCharge_ext, ip.*get(R_enlarge()),
        g_mol->maxX, g_mol->maxY, g_mol->maxZ, g_mol->centerX, g_mol->centerY,
        g_mol->centerZ, (double)maxClusterSize_ext, (double)multipole_ext,
        (double)dispersionCutoff_ext};
    int n = (int)(sizeof v / sizeof v[0]);
    for (int i = 0; i < n && i < cap; i++) out[i] = v[i];
    return n;
}

int ref_num_clusters(void) { return (int)(force().*get(R_clusterGroups())).size(); }

int ref_cluster_size(int k) { return (int)(force().*get(R_clusterGroups()))[k].size(); }

/* Cluster k: member atom indices (file order), position used by the force
 * kernels, radius, total charge, dipole[3], quadrupole[9], centre-replaced. */
void ref_get_cluster(int k, int *members, double *pos, double *radius, double *q,
                     double *dip, double *quad, int *replaced)
{
    std::forceAccel &f = force();
    const vector<int> &g = (f.*get(R_clusterGroups()))[k];
    for (size_t i = 0; i < g.size(); i++) members[i] = g[i];
    const vector3D<double> &p = (f.*get(R_clusterPos()))[k];
    pos[0] = p.X; pos[1] = p.Y; pos[2] = p.Z;
    *radius = (f.*get(R_clusterRadius()))[k];
    *q = (f.*get(R_totalCharge()))[k];
    for (int i = 0; i < 3; i++) dip[i] = (f.*get(R_dipole()))[k][i];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) quad[3 * i + j] = (f.*get(R_quadPole()))[k][i][j];
    *replaced = (f.*get(R_centerReplace()))[k] ? 1 : 0;
}

int ref_num_boundary(void)
{
    return (int)((*g_monte).*get(R_impactB()).*get(R_boundry())).size();
}

void ref_get_boundary(double *xyz)
{
    const vector<vector3D<double> > &b = (*g_monte).*get(R_impactB()).*get(R_boundry());
    for (size_t i = 0; i < b.size(); i++) {
        xyz[3 * i] = b[i].X; xyz[3 * i + 1] = b[i].Y; xyz[3 * i + 2] = b[i].Z;
    }
}

/* forceAccel::getReducedVec at n positions (forceAccel.cpp:887-908). */
void ref_force(int n, const double *pos, double *acc)
{
    std::forceAccel &f = force();
    for (int i = 0; i < n; i++) {
        vector3D<double> p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        vector3D<double> a = f.getReducedVec(p);
        acc[3 * i] = a.X; acc[3 * i + 1] = a.Y; acc[3 * i + 2] = a.Z;
    }
}

/* forceAccel::getPotential at n positions (forceAccel.cpp:943-982). */
void ref_potential(int n, const double *pos, double *u)
{
    std::forceAccel &f = force();
    for (int i = 0; i < n; i++) {
        vector3D<double> p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        u[i] = f.getPotential(p);
    }
}

/* diffEqSolver::verletVel on each (pos0, vel0), in order, one thread. */
void ref_run_list(int n, const double *pos0, const double *vel0, double *chi,
                  int *succ, int *steps, double *dE)
{
    monteTraj &m = *g_monte;
    diffEqSolver &s = m.*get(R_gasAtom());
    impactParam &ip = m.*get(R_impactB());
    for (int i = 0; i < n; i++) {
        vector3D<double> p(pos0[3 * i], pos0[3 * i + 1], pos0[3 * i + 2]);
        vector3D<double> v(vel0[3 * i], vel0[3 * i + 1], vel0[3 * i + 2]);
        localThreadParams lp;
        std::memset(&lp, 0, sizeof lp);
        double c = 0;
        bool ok = s.verletVel(dt_ext, p, v, ip.a, ip.b, ip.c, c, lp);
        chi[i] = c;
        succ[i] = ok ? 1 : 0;
        steps[i] = lp.stepCount;
        dE[i] = lp.maxErgyPctDev;
    }
}

/* monteTraj::setUpTraj (monteTraj.cpp:174-278) driven by mt19937_64(seed),
 * as thread 0 of the reference's first integral draws it
 * (monteTraj.cpp:344-349); returns the sampled (b, phi, theta, gamma, g), the
 * start state and whether the ellipsoid was hit.  rand() (gCheck) is reset
 * to srand(rand_seed); the reference never seeds it, which is srand(1). */
void ref_sample(int n, unsigned long long seed, unsigned rand_seed, double *bpgtg,
                double *pos0, double *vel0, int *hit)
{
    monteTraj &m = *g_monte;
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<double> distr(0.0, 1.0);
    std::srand(rand_seed);
    bool saved = printData_ext;
    printData_ext = true;
    for (int i = 0; i < n; i++) {
        localThreadParams lp;
        std::memset(&lp, 0, sizeof lp);
        vector3D<double> p, v;
        int idx = i;
        bool h = m.setUpTraj(0, idx, p, v, lp, gen, distr);
        bpgtg[5 * i + 0] = lp.b; bpgtg[5 * i + 1] = lp.phi; bpgtg[5 * i + 2] = lp.theta;
        bpgtg[5 * i + 3] = lp.gamma; bpgtg[5 * i + 4] = lp.g;
        pos0[3 * i] = p.X; pos0[3 * i + 1] = p.Y; pos0[3 * i + 2] = p.Z;
        vel0[3 * i] = v.X; vel0[3 * i + 1] = v.Y; vel0[3 * i + 2] = v.Z;
        hit[i] = h ? 1 : 0;
    }
    printData_ext = saved;
}

}  // extern "C"
