/*
 * uph_system.h -- drop-in entry points with the reference's own signatures.
 *
 * libuph_sph.so replaces the two translation units of the reference's
 * libSPH that hold the hot path, src/lib/derivatives.c and
 * src/lib/Search.cc, while the rest of libSPH (System.c, input.c, inputbp.c,
 * inoutflow.c, output.c) and the driver src/bin/sph.cc stay as they are.  A
 * caller relinks against it and changes nothing else.
 *
 * `System` below must have exactly the memory layout of the reference's
 * struct (src/lib/System.h:13-153) because the caller allocates it and this
 * library reads its fields: the members are declared in the same order with
 * the same types.  Only the names a reader needs are commented.
 */
#ifndef UPH_SYSTEM_H
#define UPH_SYSTEM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct __system {
  int dim;
  int *itype;
  int nx;
  int ny;
  double Lx, Ly;
  double dx, dy;
  int NumberOfInteractingParticles;
  int MaxNumberOfParticles;
  int NumberOfFluidParticles;
  int NumberOfBoundaryParticles;
  int NumberOfFixedBoundaryParticles;
  int NumberOfMovingBoundaryParticles;
  int NumberOfFrozenParticles;
  int NumberOfSolidParticles;
  int NumberOfVirtualParticles;
  int nearNeighbor;
  double LeftBoundaryPosition, LeftBoundaryVelocity, RightBoundaryPosition, LeftBoundaryAcceleration;
  double **tmp;
  double **Position;      /* [MaxN][2], contiguous behind Position[0] */
  double **Velocity;
  double **Velocity_xsph;
  double *mass;
  double *Pressure;
  double *Energy;
  double *hsml;
  double *density;
  double **Velocity_min;
  double *ddensitydt;
  double **dvdt;
  double **av;
  double *density_min;
  double density0;
  double *viscosity;
  double *ViscousStressxx, *ViscousStressxy, *ViscousStressyx, *ViscousStressyy;
  double coreCoefficient;
  double machNumber;
  double *DynamicPressure, *DynamicPressure_min, *dpdt;
  double *localDensity_min;
  double *meanCompressibility, *meanSpecDensity;
  double pressureKernelNorm;
  double *densityFluctuation, *pressureFluctuation;
  double **velocityFluctuation;
  double *normalizationFactor;
  double damping_time, tstep;
  int dampingIterations;
  double *localDensity, *localPressure, **localVelocity;
  double *wc, **dwcdx;
  double timeStep, pecletNumber, viscosity0;
  int virtualType;
  double *tempPosition, *tempPositionGate, gateVelocity;
  int printStep, screenStep;
  double lennardSelect, lidVelocity, wallViscosity;
  double totalKineticEnergy;
  int pointNeighbors;
  double pointPressure, *tempPointPressure;
  double initialEnergy, potentialEnergy;
  double *wp;
  int selectBoundaryForce;
  double springConstant0, dampingConstant0;
  double *springConstant, *dampingConstant;
  int *pj_pair;
  double *tempPointVolume;
  double **gradNormFactor;
  int flagInitSimul;
  double *localCompressibility;
  int gravityFlag;
  double *thermalDiffusivity, thermalDiffusivity0;
  int movingBoundary;
  int NumberOfInitializationSteps;
  double consistencyDensityOne, consistencyDensityTwo, consistencyDensityThree;
  double densityUncertainty;
  double *specificVolume;
  double **Position_min;
  double pressureNorm;
  double *Volume;
  double *vorticity, *approxVorticity;
  double pressureProbeX, pressureProbeY;
  double pressureProbeXX, pressureProbeYY;
  double *tempPointPressureTwo;
  int pointNeighborsTwo;
  double pointPressureTwo;
  double *xSpongeVelocity, *ySpongeVelocity;
  double *spongeFactor, spongeFactor0, spongePosition0;
  int waveAbsorption;
  double enstrophyPower;
  int stressType;
  double *specificDissipationPower, dissipationPower;
  double *specificBoundaryDissipationRate, boundaryDissipationRate;
  double *specificDissipationRate, dissipationRate, *specificDissipationRateTemp;
  int disspationControlVolume;
  double *specificTurbulentDissipationRate, *turbulentKineticEnergy;
  double *controlKineticEnergy, *controlDissipationRate, *controlMaxVelocity, *controlVolumeX;
  int controlVolumeNumber;
  int *damGateFlag;
  double *ddensitydt_approx;
  double *dpdt_approx;
  double **dvdt_approx;
  double alpha_cspline, alpha_kernelFour, alpha_deconvolutionFour, alpha_kernelFive, alpha_deconvolutionFive;
  double alpha_wendlandFour, alpha_deconvolutionSix;
  double alpha;
  double SpeedOfSound;
  double slope;
  double stroke, omega, wavePeriod;
  double eta;
  double Gravity;
  double LennardCoefficient;
  double LocalDepth, FlatBottomLength;
  double epsilon;
  int *i_pair, *j_pair;
  int *NeighborsSize;
  int *i_inflow;
  double *rij2, *w;
  double **dwdx;
  int inflowParticles;
  double CompressionFactor;
  double AdiabaticConstant;
  int niac;
  int HowManyNeighbors;
} System;

/* Replaces derivatives() of src/lib/derivatives.h:12 (derivatives.c:3137).
 * Same observable effect on the hot-path fields: the rates (ddensitydt,
 * dpdt, dvdt and their *_approx), the fluctuation fields, Pressure, the pair
 * list (i_pair, j_pair, rij2, w, dwcdx, NumberOfInteractingParticles) and
 * totalKineticEnergy / potentialEnergy.  It still calls the caller's
 * inoutflow() and inputbp() exactly where the reference does.  On an error
 * it prints the message and exits(1), the reference's own convention. */
void derivatives(System *sys, double t);

/* Replaces SearchNeighbors of src/lib/Search.cc:5 (declared at
 * derivatives.c:34-42): same arguments, same pair filter, same return value.
 * Pairs come ordered by s then j (the reference: s then libnabo heap order). */
int SearchNeighbors(const double **Position, int *i_pair, int *j_pair, double *rij2, const int NumberOfFluidParticles,
                    const int NumberOfParticles, int ParticleBoundary, const int NumberOfNeighbors, const double dist);

/* What derivatives() copies back of the pair list it computes (no
 * counterpart in the reference, whose derivatives() always fills it):
 *   2 (default) i_pair, j_pair, rij2, w, dwcdx and NumberOfInteractingParticles;
 *   1           i_pair, j_pair, rij2 and the count;
 *   0           the count only.
 * The reference's own callers (sph.cc, output.c, inputbp.c, inoutflow.c)
 * read only the count; a caller that reads none of the arrays saves their
 * device-to-host copy (40 bytes per pair) with level 0. */
void uph_dropin_set_pair_export(int level);

/* The two libSPH functions derivatives() calls back, inputbp(sys, t) and
 * inoutflow(sys) (derivatives.c:3162-3168).  By default they are the ones
 * linked with the caller (its own libSPH); a caller without a libSPH, or one
 * that loads several callers into one process, names its own here (NULL
 * restores the default).  No counterpart in the reference. */
void uph_dropin_set_callbacks(void (*inputbp_fn)(System *sys, double t), void (*inoutflow_fn)(System *sys));

#ifdef __cplusplus
}
#endif

#endif /* UPH_SYSTEM_H */
