/* C-ABI of the B200 engine for Agama's Multipole / DOP853 orbit / Staeckel-fudge action path.

   The first group of entry points has exactly the names, argument meaning and error behaviour
   of the reference's plain-C interface (src/interface_c.h), so a C/C++/Fortran/ctypes caller
   of that interface can link this library instead for the supported subset.  The remaining
   entry points are batched (many points per call) and device-pointer variants that the
   reference interface does not have; their comments name the reference routine each one
   replaces when applied point by point.

   Conventions: opaque handles are created by agama_create* and freed by agama_delete*;
   constructors return NULL on error and batched calls return 0 on success or -1 on error;
   the text of the last error of the calling thread is returned by agama_getError().
   Arrays are row-major, double precision: positions n x 3 (x,y,z), phase-space points
   n x 6 (x,y,z,vx,vy,vz), gradients n x 3, Hessians n x 6 (xx,yy,zz,xy,yz,zx).
   *Device variants take device pointers and a cudaStream_t (as void*; NULL = default stream),
   and return after enqueueing the work. */
#ifndef AGAMA_B200_H
#define AGAMA_B200_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct agama_Density agama_Density;
typedef struct agama_Potential agama_Potential;
typedef struct agama_ActionFinder agama_ActionFinder;

/* ---------------------------------------------------------------------------------------
   Entry points with the reference's names and signatures (src/interface_c.h).            */

/* reference: agama_getError, src/interface_c.h:20 (src/interface_c.cpp:25-28) */
const char* agama_getError(void);

/* reference: agama_createPotential, src/interface_c.h:45 (src/interface_c.cpp:31-51).
   Accepts "file=<coefficient file>" (optionally with "type=Multipole"): a Multipole potential
   stored by the reference's writePotential (src/potential_factory.cpp:909-930); or
   "type=Multipole, density=<model>, <model parameters>, lmax=.., gridSizeR=.., ...": a Multipole
   built from one density model (see agama_createMultipoleFromDensities). */
agama_Potential* agama_createPotential(const char* params);

/* reference: agama_deletePotential, src/interface_c.h:51 */
void agama_deletePotential(agama_Potential* potential);

/* reference: agama_evalPotential, src/interface_c.h:77 (src/interface_c.cpp:68-90):
   potential at pos, gradient into deriv[3] and Hessian into deriv2[6] when not NULL. */
double agama_evalPotential(const agama_Potential* potential, const double pos[3], double time,
    double deriv[3], double deriv2[6]);

/* reference: agama_createDensity, src/interface_c.h:35 (src/interface_c.cpp:20-29).  Density
   models (Plummer, Spheroid, ...) only serve to construct potentials, which this engine reads
   from coefficient files: always NULL, with the reason in agama_getError(). */
agama_Density* agama_createDensity(const char* params);

/* reference: agama_deleteDensity, src/interface_c.h:49 (nothing to free here) */
void agama_deleteDensity(agama_Density* density);

/* reference: agama_evalDensity, src/interface_c.h:61 (src/interface_c.cpp:63-66 ->
   Multipole::densityCyl, src/potential_multipole.cpp:1550-1559).  As in the reference, the
   object may be a potential (cast to agama_Density*): its density is the Laplacian of the
   potential / 4 pi inside the radial grid and the closed form of the power-law expansions
   outside.  NaN on failure. */
double agama_evalDensity(const agama_Density* density, const double pos[3], double time);

/* reference: agama_R_circ, src/interface_c.h:81 (src/interface_c.cpp:92-95 -> potential::R_circ,
   src/potential_utils.cpp:617-619): radius of the circular orbit of energy E in the equatorial
   plane; the potential is averaged over the azimuth if it is not axisymmetric
   (Axisymmetrized, src/potential_base.cpp:256-283, 529-590).  NaN on failure. */
double agama_R_circ(const agama_Potential* potential, double E);

/* reference: agama_R_from_Lz, src/interface_c.h:86 (potential::R_from_Lz,
   src/potential_utils.cpp:621-627): radius of the circular orbit of angular momentum Lz. */
double agama_R_from_Lz(const agama_Potential* potential, double Lz);

/* reference: agama_R_max, src/interface_c.h:91 (potential::R_max, src/potential_utils.cpp:629-631):
   the root of Phi(R, z = 0) = E. */
double agama_R_max(const agama_Potential* potential, double E);

/* reference: agama_findPlanarOrbitExtent, src/interface_c.h:104 (potential::findPlanarOrbitExtent,
   src/potential_utils.cpp:663-729): peri- and apocentre radii of the planar orbit (E, L); both
   NaN when E is outside the allowed range, both R_circ(E) when L >= L_circ(E). */
void agama_findPlanarOrbitExtent(const agama_Potential* potential, double E, double L,
    double* Rperi, double* Rapo);

/* ---------------------------------------------------------------------------------------
   Construction from arrays (reference: potential::Multipole(gridRadii, Phi, dPhi),
   src/potential_multipole.cpp:1491-1516, the constructor behind the coefficient file).
   radii[gridSizeR] increasing; Phi and dPhi are numCoefs x gridSizeR with the coefficient
   index c = l*(l+1)+m, numCoefs = (lmax+1)^2. */
agama_Potential* agama_createMultipoleFromCoefs(int gridSizeR, const double* radii, int numCoefs,
    const double* Phi, const double* dPhi);

/* A Multipole built from density models: the Poisson solve of the reference's createMultipole
   (src/potential_multipole.cpp:1400-1441; chooseGridRadii :369-484, computePotentialCoefsFromSource
   :1013-1114, restrictSphHarmCoefs :151-185) for the sum of the given densities, each a key=value
   string as the reference's createDensity takes it (type=Dehnen | Plummer | NFW | MiyamotoNagai |
   Spheroid | Disk, with mass, scaleRadius, gamma, axisRatioY, axisRatioZ, scaleHeight, alpha,
   beta, densityNorm, surfaceDensity, outerCutoffRadius, cutoffStrength as they apply);
   multipoleParams: lmax, mmax, gridSizeR, rmin, rmax (0 = chosen from the density), symmetry,
   fixOrder.  agama_createPotential accepts the single-density form "type=Multipole,
   density=<type>, ..." of the reference's plain-C interface (src/interface_c.cpp:31-51). */
agama_Potential* agama_createMultipoleFromDensities(const char* multipoleParams, int numComponents,
    const char* const* densityParams);

/* The same Poisson solve on the host only (no device): the coefficients that
   agama_createMultipoleFromDensities builds the potential from.  Call with radii == NULL to get
   gridSizeR and numCoefs; then radii[gridSizeR], Phi and dPhi[numCoefs x gridSizeR] (index
   c = l*(l+1)+m, as agama_createMultipoleFromCoefs takes them). */
int agama_multipoleCoefsFromDensities(const char* multipoleParams, int numComponents,
    const char* const* densityParams, int* gridSizeR, int* numCoefs, double* radii, double* Phi, double* dPhi);

/* order, symmetry (coord::SymmetryType bit mask) and grid sizes of a Multipole potential */
int agama_getPotentialInfo(const agama_Potential* potential, int* lmax, int* mmax, int* symmetry,
    int* gridSizeR, int* gridSizeTau);

/* Host-only check of a coefficient file: parses it and builds the tables without a device
   (reference: the parsing half of createPotential for type=Multipole,
   src/potential_factory.cpp:725-746).  Returns 0 and the order / symmetry / grid sizes. */
int agama_inspectMultipoleFile(const char* file, int* lmax, int* mmax, int* symmetry,
    int* gridSizeR, int* gridSizeTau);

/* reference: writePotential(fileName, potential), src/potential_factory.h:290-300, which for a
   Multipole writes writePotentialMultipole's text (src/potential_factory.cpp:909-930): the
   coefficient file of a potential, readable by the reference's readPotential / createPotential
   and by agama_createPotential("file=...").  Numbers are written with 17 significant digits
   (the reference writes 11-22), so the file reproduces the potential's coefficients exactly. */
int agama_writePotential(const char* fileName, const agama_Potential* potential);

/* The same file from coefficient arrays (layout as agama_createMultipoleFromCoefs), host-only:
   no device is needed. */
int agama_writeMultipoleCoefs(const char* fileName, int gridSizeR, const double* radii, int numCoefs,
    const double* Phi, const double* dPhi);

/* Batched potential / gradient / Hessian at n points, host buffers (any output may be NULL).
   Replaces n calls of agama_evalPotential (src/interface_c.cpp:68-90); the reference batches
   the same call in Python, BatchFunction over BasePotential::eval (src/interface_python.cpp:1405-1485,
   :3077-3104). */
int agama_evalPotentialMany(const agama_Potential* potential, long n, const double* pos, double time,
    double* phi, double* deriv, double* deriv2);

/* The same on device buffers, enqueued on the given stream. */
int agama_evalPotentialManyDevice(const agama_Potential* potential, long n, const double* pos,
    double* phi, double* deriv, double* deriv2, void* stream);

/* Batched potential / gradient / Hessian at n cylindrical points, host buffers: pos is n x 3 in the
   order (R, z, phi) of the reference's coord::PosCyl; deriv n x 3 (dR, dz, dphi) as coord::GradCyl;
   deriv2 n x 6 (dR2, dz2, dphi2, dRdz, dzdphi, dRdphi) as coord::HessCyl.  Replaces n calls of
   BasePotential::eval(PosCyl, ...), which a Multipole answers natively in cylindrical coordinates
   (BasePotentialCyl::evalCyl, src/potential_base.h:237-262; Multipole::evalCyl,
   src/potential_multipole.cpp:1538-1548). */
int agama_evalPotentialCylMany(const agama_Potential* potential, long n, const double* pos, double time,
    double* phi, double* deriv, double* deriv2);

/* The same on device buffers, enqueued on the given stream. */
int agama_evalPotentialCylManyDevice(const agama_Potential* potential, long n, const double* pos,
    double* phi, double* deriv, double* deriv2, void* stream);

/* Batched density of a potential at n points (n x 3), host buffers: n calls of agama_evalDensity
   (the reference's Python Density.density batches the same, src/interface_python.cpp:2439). */
int agama_evalDensityMany(const agama_Potential* potential, long n, const double* pos, double time,
    double* rho);

/* The same on device buffers, enqueued on the given stream. */
int agama_evalDensityManyDevice(const agama_Potential* potential, long n, const double* pos, double* rho,
    void* stream);

/* Batched radius queries, one per item, host buffers: query 0 = R_circ(in1 = E), 1 = R_from_Lz
   (in1 = Lz), 2 = R_max(in1 = E): radius into out1 (in2, out2 unused, may be NULL);
   3 = findPlanarOrbitExtent(in1 = E, in2 = L): pericentre into out1, apocentre into out2.
   Replaces n calls of agama_R_circ / agama_R_from_Lz / agama_R_max / agama_findPlanarOrbitExtent
   (the reference batches them in Python as Potential.Rcirc / Rmax / Rperiapo,
   src/interface_python.cpp:3354-3512). */
int agama_potentialRadiiMany(const agama_Potential* potential, int query, long n, const double* in1,
    const double* in2, double* out1, double* out2);

/* The same on device buffers, enqueued on the given stream. */
int agama_potentialRadiiManyDevice(const agama_Potential* potential, int query, long n, const double* in1,
    const double* in2, double* out1, double* out2, void* stream);

/* ---------------------------------------------------------------------------------------
   Orbit integration (DOP853).  Each of the n orbits starts at ic[i] (x,y,z,vx,vy,vz, in the
   frame rotating with pattern speed Omega about z) at time 0 and is integrated for time T[i]
   with relative accuracy `accuracy` and at most maxNumSteps accepted steps (<= 0: 1e8).
   Outputs: the final point in the rotating frame, the number of accepted steps and a status
   (0 ok, 1 step limit reached, 2 zero / non-finite step, 3 non-finite error estimate).
   Replaces n runs of orbit::OrbitIntegrator<Car>(pot, Omega, {accuracy, maxNumSteps}).init(ic)
   + run(T) with a final-point RuntimeTrajectory (src/orbit.h:165-315, src/orbit.cpp:15-117),
   as driven by the reference's Python orbit() (src/interface_python.cpp:8101-8160). */
int agama_integrateOrbitsMany(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, int* status);

/* Lanes of a warp that integrate one orbit together (no reference counterpart): 1, 2, 4 or 8
   (the lanes share the spline evaluations of potentials with up to 8 azimuthal harmonics; other
   potentials use 1), or 0 (default) to let the library choose: a timing trial on the batch's
   first orbits, once per device, potential and batch-size class, then cached.  The trial runs on
   the caller's stream and waits for it, so the first call of a class should not be made during
   stream capture.  Applies to the orbit entry points below except the allocation-free one. */
int agama_setOrbitLanesPerOrbit(int lanes);

/* Threads per block of the orbit kernels (no reference counterpart): 32, 64 or 128, or 0
   (default) to let the library choose together with the lanes per orbit, by the same timing trial
   (every lane count times every block size).  Neither setting changes any result bit. */
int agama_setOrbitBlockSize(int block);

/* Mixed precision for orbit batches (no reference counterpart): 1 evaluates the non-axisymmetric
   (m != 0) harmonics of multi-harmonic Multipole potentials from an FP32 copy of the spline table,
   with the radial m = 0 part, the azimuthal sums, the integrator state, its stages and its error
   norm in FP64; 0 (default) is all FP64.  Forces then differ from FP64 by about 1e-7 of the
   non-axisymmetric part, and final states of regular orbits by the growth of that over the
   integration (the Python orbit_precision_error helper measures it per orbit).  One lane per orbit
   in mixed mode; other potentials and the allocation-free entry point stay FP64.  Applies to
   batches launched or captured afterwards. */
int agama_setOrbitPrecision(int mixed);

/* Runtime functions of orbits: a target that accumulates each orbit's time-weighted samples into
   the basis elements of a classic spheroidal density grid.  reference: galaxymodel::
   TargetDensityClassic<degree> (src/galaxymodel_densitygrid.h:66-108, :149-238) as created by the
   Python Target(type='DensityClassicTopHat' (degree 0) or 'DensityClassicLinear' (degree 1),
   gridr, stripsPerPane, axisRatioY, axisRatioZ) (src/interface_python.cpp:7185-7205), attached to
   each orbit by RuntimeFncTarget (src/galaxymodel_target.h:99-150; Python orbit(targets=...),
   src/interface_python.cpp:8114-8121).  gridr: gridSize increasing radii (a leading 0 is
   dropped); NULL with agama_getError() on invalid parameters. */
typedef struct agama_Target agama_Target;
agama_Target* agama_createTargetDensityClassic(int degree, int stripsPerPane, int gridSize, const double* gridr,
    double axisRatioY, double axisRatioZ);
void agama_deleteTarget(agama_Target* target);
/* number of basis elements (values recorded per orbit) */
int agama_targetNumCoefs(const agama_Target* target);

/* Orbits as agama_integrateOrbitsManyDevice (work queue) with the target's runtime function:
   every accepted step adds 10 points of its dense output, at the middles of equal sub-steps and
   in the frame of the potential, each weighted by the sub-step's duration, to the orbit's row;
   at the end the row is converted to FP32 and divided by the integration time
   (RuntimeFncTarget::processTimestep and its destructor).  output: n x numCoefs floats. */
int agama_integrateOrbitsTargetManyDevice(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, const agama_Target* target, float* output,
    double* finalState, long* numSteps, int* status, void* stream);
/* The same on host buffers (finalState, numSteps, status may be NULL). */
int agama_integrateOrbitsTargetMany(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, const agama_Target* target, float* output,
    double* finalState, long* numSteps, int* status);

/* An orbit batch captured once in a CUDA graph (no reference counterpart): the work-counter reset
   and the persistent DOP853 kernel over the given device buffers, with the lanes per orbit and
   the block size settled (autotuner trial) before the capture.  Each agama_orbitGraphLaunch replays the batch on the
   stream, reading the current contents of ic and T: with finalState == ic every launch continues
   the orbits for another T (each orbit reads its start before writing its end).  The buffers
   must stay valid while the graph exists. */
typedef struct agama_OrbitGraph agama_OrbitGraph;
agama_OrbitGraph* agama_orbitGraphCreate(const agama_Potential* potential, long n, const double* ic, const double* T,
    double Omega, double accuracy, long maxNumSteps, double* finalState, long* numSteps, long* numRejected,
    int* status);
int agama_orbitGraphLaunch(agama_OrbitGraph* graph, void* stream);
int agama_orbitGraphLanes(const agama_OrbitGraph* graph);
int agama_orbitGraphBlockSize(const agama_OrbitGraph* graph);
void agama_orbitGraphDelete(agama_OrbitGraph* graph);

/* Orbits with their trajectories sampled at trajSize (>= 2) regular times t_k = k T/(trajSize-1)
   of each orbit (the reference's RuntimeTrajectory with sampling interval T/(trajSize-1), as
   its Python orbit(trajsize=...), src/orbit.cpp:15-47: 7th-order dense output of the DOP853 steps,
   src/math_ode.cpp:381-426); traj is n x trajSize x 6 in the frame rotating with Omega, NaN where
   an orbit produced no sample (stopped early); T = 0 gives the start as samples 0 and 1.
   Device-pointer and host-buffer variants; finalState, numSteps, status as for
   agama_integrateOrbitsMany (in the host variant finalState may be NULL). */
int agama_integrateOrbitsTrajectoryManyDevice(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, int trajSize, double* traj,
    double* finalState, long* numSteps, int* status, void* stream);
int agama_integrateOrbitsTrajectoryMany(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, int trajSize, double* traj,
    double* finalState, long* numSteps, int* status);

/* The same on device buffers (numSteps, numRejected, status may be NULL; numRejected counts
   rejected step attempts).  useQueue != 0 drains the batch from a device work queue with a
   grid sized to the GPU (for batches of very uneven integration times). */
int agama_integrateOrbitsManyDevice(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, long* numRejected, int* status, int useQueue, void* stream);

/* The same work-queue batch (as agama_integrateOrbitsManyDevice with useQueue != 0), but the
   library allocates nothing: no cudaMalloc, cudaFree or allocating library routine runs.  It is
   for callers that cannot let a library allocate device memory -- applications whose memory
   manager has reserved (nearly) all of the GPU's memory up front, latency-critical loops in which
   an allocation would synchronise the device and stall other streams, and plugin hosts that
   account for every byte of device memory.  This entry point has no counterpart in the reference.
   The queue counter lives in a static array of 32 counters (256 bytes) in device memory, held by
   every GPU that loads the library until the process exits; queueSlot (0..31) selects one, and a
   value outside that range is rejected with an error.  Each call clears its counter on `stream`
   before the launch; the array keeps the last call's values.  Calls that overlap on the GPU and
   use the same slot race (orbits may be skipped or integrated twice): give batches that may run
   at the same time different slots.  The first call on each device looks up the array's device
   address (cudaGetSymbolAddress) -- make that first call before any stream capture.
   It always integrates in FP64 with one lane per orbit: agama_setOrbitPrecision and
   agama_setOrbitLanesPerOrbit do not apply to it (with mixed precision switched on, its results
   are those of the FP64 batch, not those of agama_integrateOrbitsManyDevice). */
int agama_integrateOrbitsManyDeviceNoAlloc(const agama_Potential* potential, long n, const double* ic,
    const double* T, double Omega, double accuracy, long maxNumSteps, double* finalState,
    long* numSteps, long* numRejected, int* status, int queueSlot, void* stream);

/* Mixed precision for the Staeckel-fudge action integrals (no reference counterpart): 1 computes
   the integrand after F(tau) (p^2 = F / (2 (tau - Delta^2)^2 tau), its square root, the
   end-point stretch) and the Gauss-Legendre sums in FP32, the sums compensated (Kahan), while the
   potential, F(tau), the integrals of motion and the turning-point root searches stay FP64;
   0 (default) is all FP64.  The actions then differ from FP64 by about 1e-7 relative.  Applies to
   the action entry points without angles / frequencies called afterwards. */
int agama_setActionPrecision(int mixed);

/* ---------------------------------------------------------------------------------------
   Staeckel-fudge actions (axisymmetric potentials only).  posvel: n x 6 Cartesian points;
   act: n x 3 (Jr, Jz, Jphi); unbound points (E >= 0) give Jr = Jz = NaN, as in the reference
   (src/actions_staeckel.cpp:648-656). */

/* reference: agama_createActionFinder, src/interface_c.h:113 (src/interface_c.cpp:113-123):
   the Staeckel-fudge action finder of an axisymmetric potential, with its focal-distance table
   built from shell orbits on the device (ActionFinderAxisymFudge constructor,
   src/actions_staeckel.cpp:751-795) and its L_circ(E) interpolator (potential::Interpolator,
   src/potential_utils.cpp:757-870).  NULL (with agama_getError) for non-axisymmetric potentials. */
agama_ActionFinder* agama_createActionFinder(const agama_Potential* potential);

/* sizes and contents of an action finder's tables (layout as agama_createActionFinderFromTables) */
int agama_getActionFinderTableSizes(const agama_ActionFinder* actionFinder, int* nE, int* nL, int* nLofE,
    int* nRofL, int* nPhiofR);
int agama_getActionFinderTables(const agama_ActionFinder* actionFinder, double* gridE, double* gridL,
    double* delta, double* LofE, double* RofL, double* PhiofR, double* scalars);

/* reference: agama_deleteActionFinder, src/interface_c.h:118 */
void agama_deleteActionFinder(agama_ActionFinder* actionFinder);

/* reference: agama_evalActionsAnglesFrequencies, src/interface_c.h:135 (src/interface_c.cpp:129-155):
   actions, angles and frequencies of one point through the action finder (any output pointer
   may be NULL); NaN in every output when the call fails, with the message in agama_getError(). */
void agama_evalActionsAnglesFrequencies(const agama_ActionFinder* actionFinder, const double posvel[6],
    double actions[3], double angles[3], double frequencies[3]);

/* reference: agama_evalActionsAnglesFrequenciesStandalone, src/interface_c.h:155
   (src/interface_c.cpp:157-192): actions, angles and frequencies of one point for a given focal
   distance fd (actions::evalAxisymFudge, src/actions_staeckel.cpp:683-693). */
void agama_evalActionsAnglesFrequenciesStandalone(const agama_Potential* potential, double fd,
    const double posvel[6], double actions[3], double angles[3], double frequencies[3]);

/* An action finder from precomputed tables: the focal-distance grid Delta(scaledE, chi) of
   ActionFinderAxisymFudge (gridE[nE] = ln(1/Phi0 - 1/E), gridL[nL] = chi = s(Lz/Lcirc),
   delta[nE x nL]; src/actions_staeckel.cpp:751-795) and the L_circ(E) interpolator of
   potential::Interpolator (quintic splines LofE, RofL, PhiofR stored as [x | f | f' | f''] with
   n nodes each; scalars = {1/Phi0 of the finder, 1/Phi0 of the interpolator, slopeOut,
   coefOut, massOut}; src/potential_utils.cpp:757-980). */
agama_ActionFinder* agama_createActionFinderFromTables(const agama_Potential* potential,
    int nE, const double* gridE, int nL, const double* gridL, const double* delta,
    int nLofE, const double* LofE, int nRofL, const double* RofL, int nPhiofR, const double* PhiofR,
    const double* scalars);

/* Batched actions through the action finder, host buffers; fdOut (n, may be NULL) receives the
   focal distance used for each point.  Replaces n calls of agama_evalActionsAnglesFrequencies
   / ActionFinderAxisymFudge::eval (src/actions_staeckel.cpp:954-979) as batched by the
   reference's Python ActionFinder (src/interface_python.cpp:3761-3822). */
int agama_evalActionsMany(const agama_ActionFinder* actionFinder, long n, const double* posvel,
    double* act, double* fdOut);

/* The same on device buffers. */
int agama_evalActionsManyDevice(const agama_ActionFinder* actionFinder, long n, const double* posvel,
    double* act, double* fdOut, void* stream);

/* Batched actions for given focal distances fd[n] (or fd0 for all points when fd is NULL);
   replaces n calls of agama_evalActionsAnglesFrequenciesStandalone. */
int agama_evalActionsStandaloneMany(const agama_Potential* potential, long n, const double* posvel,
    const double* fd, double fd0, double* act);

/* The same on device buffers; rootIters (n, may be NULL) receives the number of root-finder
   iterations spent on each point. */
int agama_evalActionsStandaloneManyDevice(const agama_Potential* potential, long n, const double* posvel,
    const double* fd, double fd0, double* act, int* rootIters, void* stream);

/* Batched actions, angles (theta_r, theta_z, theta_phi) and frequencies (Omega_r, Omega_z,
   Omega_phi) through the action finder, host buffers of n x 3 each; any of act / ang / freq may
   be NULL (not all three).  Replaces n calls of agama_evalActionsAnglesFrequencies
   (actions::evalAxisym, src/actions_staeckel.cpp:645-670, batched as by the reference's Python
   ActionFinder with angles / frequencies, src/interface_python.cpp:3761-3822). */
int agama_evalActionsAnglesFrequenciesMany(const agama_ActionFinder* actionFinder, long n,
    const double* posvel, double* act, double* ang, double* freq);

/* The same on device buffers. */
int agama_evalActionsAnglesFrequenciesManyDevice(const agama_ActionFinder* actionFinder, long n,
    const double* posvel, double* act, double* ang, double* freq, void* stream);

/* Batched actions, angles and frequencies for given focal distances fd[n] (or fd0 for all
   points when fd is NULL); replaces n calls of agama_evalActionsAnglesFrequenciesStandalone. */
int agama_evalActionsAnglesFrequenciesStandaloneMany(const agama_Potential* potential, long n,
    const double* posvel, const double* fd, double fd0, double* act, double* ang, double* freq);

/* The same on device buffers. */
int agama_evalActionsAnglesFrequenciesStandaloneManyDevice(const agama_Potential* potential, long n,
    const double* posvel, const double* fd, double fd0, double* act, double* ang, double* freq, void* stream);

/* ---------------------------------------------------------------------------------------
   Learned root brackets of the action finder (no reference counterpart): a network trained on the
   finder's own root searches predicts nu_max, lambda_min and lambda_max of each point; each
   search then runs on its plain bracket with the plain tolerance but takes the predicted root as
   its first iterate, and its root is checked by one evaluation beyond it (a failed check hands the
   limit to the plain search); points predicted near the focal line keep the plain searches, so the
   actions keep the finder's accuracy (1e-6 of the plain searches' actions).

   agama_actionFinderBracketSamples: the network's inputs (n x 6: the point's E, Lz, R, z, vR, vz
   in scale-free form: ln r, |z|/r, vR/v_esc, vz sign(z)/v_esc, |vphi|/v_esc with v_esc =
   sqrt(-2 Phi), ln(Delta/r)) and targets (n x 3, fractions in [0, 1]: (nu_max - |nu|)/(Delta^2 -
   |nu|), (lambda_min - Delta^2)/(lambda - Delta^2), (lambda - Delta^2)/(lambda_max - Delta^2))
   with 0/1 masks of the limits that needed a search, from the plain searches of n points (host
   buffers).
   agama_actionFinderTrainBrackets: trains a new network on n points (90 % training, 10 % to size
   the brackets: half-width = twice the 95th percentile of the held-out error, reported in
   widths[3]), attaches it and switches it on; lossHistory (epochs floats) may be NULL.
   agama_actionFinderUseBrackets: switches the trained predictor on or off.
   agama_actionFinderBracketStats: {root searches, searches started from a predicted root, failed
   checks (plain searches after them), root-finder iterations} since the last reset.
   agama_actionFinderCountBrackets: keeps (1, the default once a network is trained) or stops (0)
   those counters; without them the searches run in a kernel compiled without the counters. */
int agama_actionFinderBracketSamples(const agama_ActionFinder* actionFinder, long n, const double* posvel,
    float* features, float* target, float* mask);
int agama_actionFinderTrainBrackets(agama_ActionFinder* actionFinder, long n, const double* posvel, int epochs,
    int batch, float lr, unsigned long long seed, float* lossHistory, float* widths);
/* the trained network's predictions (n x 3, in the target units above) for given inputs (n x 6) */
int agama_actionFinderPredictBrackets(const agama_ActionFinder* actionFinder, long n, const float* features,
    float* prediction);
int agama_actionFinderUseBrackets(agama_ActionFinder* actionFinder, int on);
int agama_actionFinderBracketStats(agama_ActionFinder* actionFinder, long long* stats, int reset);
int agama_actionFinderCountBrackets(agama_ActionFinder* actionFinder, int on);

/* ---------------------------------------------------------------------------------------
   Tensor-core GEMM of the bracket-predictor network (no reference counterpart; the reference has
   no learned part): C[M x N] (FP32, leading dimension ldc) = A[M x K] * B[N x K]^T, plus the old C
   when accumulate is non-zero.  A and B are BF16 row-major with K contiguous, device pointers
   aligned to 16 bytes; M and N multiples of 128, K a multiple of 64.  Asynchronous on stream. */
int agama_gemmBf16Device(int M, int N, int K, const void* A, const void* B, float* C, int ldc,
    int accumulate, void* stream);

/* ---------------------------------------------------------------------------------------
   Bracket-predictor network (no reference counterpart; the reference has no learned part):
   6 -> 128 -> 128 -> 128 -> 3 with SiLU, BF16 weights in the hidden products on the tensor cores,
   FP32 master parameters, Adam.  Parameters (agama_mlpNumParams() floats): W1[128x6] b1
   W2[128x128] b2 W3[128x128] b3 W4[3x128] b4, weights row-major [out][in]; scaling (18 floats):
   input mean[6], input std[6], output mean[3], output std[3]. */
typedef struct agama_Mlp agama_Mlp;
agama_Mlp* agama_mlpCreate(unsigned long long seed);
void agama_mlpDelete(agama_Mlp* net);
int agama_mlpNumParams(void);
int agama_mlpGetParams(const agama_Mlp* net, float* params, float* scaling);
int agama_mlpSetParams(agama_Mlp* net, const float* params, const float* scaling);
/* loss (masked mean squared error) and gradient (host output) of one batch of STANDARDISED inputs
   x[batch x 6], targets t[batch x 3] and masks (0/1) [batch x 3]; batch a multiple of 128 */
int agama_mlpLossGrad(agama_Mlp* net, int batch, const float* x, const float* t, const float* mask,
    float* grad, float* loss);
/* Adam training on n raw samples (the standardisation is derived from them and kept); lossHistory
   (epochs floats, may be NULL) receives the mean loss of each epoch; batch a multiple of 128 */
int agama_mlpTrain(agama_Mlp* net, long n, const float* x, const float* t, const float* mask, int epochs,
    int batch, float lr, unsigned long long seed, float* lossHistory);
/* predictions y[n x 3] (raw units) for raw inputs x[n x 6], device pointers, on stream: the fused
   tensor-core inference kernel */
int agama_mlpPredictDevice(const agama_Mlp* net, long n, const float* x, float* y, void* stream);
/* synchronises and reports whether an inference kernel of this network gave up waiting for its
   tensor cores */
int agama_mlpCheck(const agama_Mlp* net);

/* ---------------------------------------------------------------------------------------
   Measurement helper (no reference counterpart): FP64 fused-multiply-add throughput of the
   current device in TFLOP/s, measured with independent FMA chains; the roofline denominator
   of the FP64-bound kernels above. */
int agama_measureFP64Throughput(double* tflops);

/* Phase timing of the action computation (no reference counterpart): on = 1 clears and starts
   recording CUDA events around the phases of every later action call (on the call's stream);
   on = 0 stops, waits for the recorded events and returns in ms[4] the summed device durations of
   the phases (prepare, bracket-network inference, root searches, integrals / angles) and in
   *passes the number of passes timed (ms, passes may be null). */
int agama_actionPhaseTiming(int on, double* ms, long* passes);

#ifdef __cplusplus
}
#endif
#endif
