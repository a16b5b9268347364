/*
 * icempm_oracle.c -- FP64 CPU restatement of the reference MPM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check and the benchmark's CPU-baseline leg may load it; the product path
 * (the CUDA library) never does.
 *
 * It restates, in plain C with OpenMP, the semantics of igorg520b/iceMPM_2d_sp
 *   simulation/kernels.cuh          P2G (39-104), grid update (109-177),
 *                                   G2P (181-315), helpers (323-566)
 *   simulation/helper_math.cuh      polar decomposition (24-44), 2x2 SVD (78-143)
 *   simulation/givens.cuh           Givens fill / rotation / compose (117-154, 190-197)
 *   simulation/parameters_sim.cpp   ComputeLame / ComputeHelperVariables (122-140)
 *   simulation/model.cpp            sub-step order (18-39)
 *   simulation/hssoa/host_side_soa.cpp  RemoveDisabledAndSort (36-47)
 * in FP64, on the reference HSSOA layout (19 rows x capacity doubles) and the
 * reference grid layout (9 rows x pitch doubles, node = y + x*GridY).
 *
 * Eigen 2x2 arithmetic in the reference (determinant, products, norm,
 * normalized) is written out with the same operand order Eigen uses for
 * fixed-size 2x2 expressions; normalized() of a zero vector returns the
 * vector unchanged (Eigen >= 3.3 behaviour).
 *
 * P2G is deterministic and independent of the thread count: points are
 * bucketed into strips of 4 grid columns; even strips are scattered in one
 * parallel pass and odd strips in a second (a 3x3 stencil never reaches two
 * strips of the same colour), each strip in point-index order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/icempm.h"

typedef icempm_simparams_t SP;

static const double coeff1 = 1.4142135623730950;     /* kernels.cuh:7 */
static const double coeff1_inv = 0.7071067811865475; /* kernels.cuh:8 */

/* ---- uint32 stored in the low 4 bytes of a double slot (little endian) -- */
static inline uint32_t slot_u32(const double *p) { uint32_t v; memcpy(&v, p, 4); return v; }
static inline void slot_set_u32(double *p, uint32_t v) { memcpy(p, &v, 4); }

/* ---------------- parameters_sim.cpp:122-140 ---------------------------- */
void orc_compute_helpers(SP *p)
{
    p->ParticleMass = p->ParticleVolume * p->IceDensity;
    p->UpdateEveryNthStep = (int)(p->AnimationFramePeriod / p->InitialTimeStep);
    p->cellsize_inv = 1. / p->cellsize;
    p->Dp_inv = 4. / (p->cellsize * p->cellsize);
    p->dt_vol_Dpinv = p->InitialTimeStep * p->ParticleVolume * p->Dp_inv;
    p->vmax = 0.25 * p->cellsize / p->InitialTimeStep;
    p->lambda = p->YoungsModulus * p->PoissonsRatio / ((1 + p->PoissonsRatio) * (1 - 2 * p->PoissonsRatio));
    p->mu = p->YoungsModulus / (2 * (1 + p->PoissonsRatio));
    p->kappa = p->mu * 2. / 3. + p->lambda;
}

/* Defaults of SimParams::Reset (parameters_sim.cpp:7-55). */
void orc_reset_params(SP *p)
{
    memset(p, 0, sizeof(*p));
    p->nPartitions = 1;
    p->SnapshotPeriod = 25;
    p->windDragCoeff_airDensity = 0.0025 * 1.2;
    p->waterDragEffectiveLinear = 0.01;
    p->waterDragEffectiveQuadratic = 0.01;
    p->InitialTimeStep = 3.e-5;
    p->YoungsModulus = 5.e8;
    p->ParticleViewSize = 2.5f;
    p->sea_water_density = 1030;
    p->SimulationEndTime = 20000;
    p->AnimationFramePeriod = 200;
    p->PoissonsRatio = 0.3;
    p->IceDensity = 916;
    p->IceCompressiveStrength = 100e6;
    p->IceTensileStrength = 10e6;
    p->IceShearStrength = 1e6;
    p->IceTensileStrength2 = 10e6;
    p->RidgeFormationCoeff = 30;
    p->DP_phi = 62;
    p->DP_threshold_p = 1e4;
    p->tpb_P2G = 256;
    p->tpb_Upd = 512;
    p->tpb_G2P = 128;
    /* cellsize is 0 until a grid is loaded; ComputeHelperVariables then gives inf
       helpers exactly as the reference does; callers set cellsize first. */
}

/* ---------------- 2x2 helpers (row-major m[0]=m00 m[1]=m01 m[2]=m10 m[3]=m11) */
static inline double det2(const double *m) { return m[0] * m[3] - m[2] * m[1]; }
static inline void mul2(const double *a, const double *b, double *c)
{
    double r0 = a[0] * b[0] + a[1] * b[2];
    double r1 = a[0] * b[1] + a[1] * b[3];
    double r2 = a[2] * b[0] + a[3] * b[2];
    double r3 = a[2] * b[1] + a[3] * b[3];
    c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
static inline void mul2_abt(const double *a, const double *b, double *c) /* a*b^T */
{
    double r0 = a[0] * b[0] + a[1] * b[1];
    double r1 = a[0] * b[2] + a[1] * b[3];
    double r2 = a[2] * b[0] + a[3] * b[1];
    double r3 = a[2] * b[2] + a[3] * b[3];
    c[0] = r0; c[1] = r1; c[2] = r2; c[3] = r3;
}
/* dev(A) = A - tr(A)/2 I (kernels.cuh:518-521) */
static inline void dev2(const double *a, double *d)
{
    double t = (a[0] + a[3]) / 2;
    d[0] = a[0] - t; d[1] = a[1]; d[2] = a[2]; d[3] = a[3] - t;
}
/* Frobenius norm, Eigen column-major summation order */
static inline double norm2(const double *a)
{
    return sqrt(a[0] * a[0] + a[2] * a[2] + a[1] * a[1] + a[3] * a[3]);
}

/* CalculateWeightCoeffs (kernels.cuh:323-332): ww[k][d], k = node offset+1 */
void orc_weights(const double pos[2], double ww[3][2])
{
    for (int d = 0; d < 2; d++) {
        double v0 = 0.5 - pos[d], v1 = pos[d], v2 = pos[d] + 0.5;
        ww[0][d] = 0.5 * v0 * v0;
        ww[1][d] = 0.75 - v1 * v1;
        ww[2][d] = 0.5 * v2 * v2;
    }
}

/* KirchhoffStress_Wolper (kernels.cuh:525-535) */
void orc_kirchhoff(const SP *p, const double F[4], double PFt[4])
{
    double Je = det2(F);
    double b[4], db[4];
    mul2_abt(F, F, b);
    dev2(b, db);
    double a = p->mu * (1. / Je);
    double c = p->kappa * 0.5 * (Je * Je - 1.);
    PFt[0] = a * db[0] + c;
    PFt[1] = a * db[1];
    PFt[2] = a * db[2];
    PFt[3] = a * db[3] + c;
}

/* ComputePQ (kernels.cuh:337-343) */
void orc_compute_pq(const SP *p, const double F[4], double *Je, double *pp, double *qq)
{
    *Je = det2(F);
    *pp = -(p->kappa / 2.) * ((*Je) * (*Je) - 1.);
    double b[4], db[4];
    mul2_abt(F, F, b);
    dev2(b, db);
    *qq = coeff1 * p->mu * (1. / (*Je)) * norm2(db);
}

/* svd2x2 (kernels.cuh:486-499) over singular_value_decomposition and
 * polar_decomposition (helper_math.cuh:24-44, 78-143) with GivensRotation
 * (givens.cuh:117-154, 190-197).  F is row-major; U, V are returned
 * row-major as the reference's Eigen comma-initialiser leaves them:
 * U = [[cu, su], [-su, cu]], V = [[cv, sv], [-sv, cv]]. */
void orc_svd2x2(const double F[4], double U[4], double S[2], double V[4])
{
    /* Eigen data() is column-major */
    double a[4] = {F[0], F[2], F[1], F[3]};
    /* polar decomposition */
    double x0 = a[0] + a[3], x1 = a[1] - a[2];
    double den = sqrt(x0 * x0 + x1 * x1);
    double uc = 1, us = 0;
    if (den != 0) { uc = x0 / den; us = -x1 / den; }
    double s[4] = {a[0], a[1], a[2], a[3]};
    for (int d = 0; d < 2; d++) { /* mat_rotation<2> rows 0,1 */
        double t1 = s[0 + d * 2], t2 = s[1 + d * 2];
        s[0 + d * 2] = uc * t1 - us * t2;
        s[1 + d * 2] = us * t1 + uc * t2;
    }
    double cosine, sine, sig0, sig1;
    double x = s[0], y = s[2], z = s[3];
    double y2 = y * y;
    if (y2 == 0) {
        cosine = 1; sine = 0; sig0 = x; sig1 = z;
    } else {
        double tau = 0.5 * (x - z);
        double w = sqrt(tau * tau + y2);
        double t = (tau > 0) ? y / (tau + w) : y / (tau - w);
        cosine = 1. / sqrt(t * t + 1.);
        sine = -t * cosine;
        double c2 = cosine * cosine;
        double csy = 2 * cosine * sine * y;
        double s2 = sine * sine;
        sig0 = c2 * x - csy + s2 * z;
        sig1 = s2 * x + csy + c2 * z;
    }
    double vc, vs;
    if (sig0 < sig1) {
        double tmp = sig0; sig0 = sig1; sig1 = tmp;
        vc = -sine; vs = cosine;
    } else {
        vc = cosine; vs = sine;
    }
    /* u *= v */
    double nc = uc * vc - us * vs;
    double ns = us * vc + uc * vs;
    uc = nc; us = ns;
    /* fill<2> gives column-major {c, s, -s, c}; mU << U[0..3] reads it row-major */
    U[0] = uc; U[1] = us; U[2] = -us; U[3] = uc;
    V[0] = vc; V[1] = vs; V[2] = -vs; V[3] = vc;
    S[0] = sig0; S[1] = sig1;
}

/* GetParametersForGrain (kernels.cuh:538-566) */
static void grain_params(const SP *p, double *pmin, double *pmax, double *qmax,
                         double *beta, double *mSq, double *pmin2)
{
    *pmax = p->IceCompressiveStrength;
    *pmin = -p->IceTensileStrength;
    *qmax = p->IceShearStrength * 1.0;
    *pmin2 = -p->IceTensileStrength2 * 1.0;
    *beta = p->IceTensileStrength / p->IceCompressiveStrength;
    *mSq = (4. * (*qmax) * (*qmax) * (1. + 2. * (*beta))) / (((*pmax) - (*pmin)) * ((*pmax) - (*pmin)));
}

/* CheckIfPointIsInsideFailureSurface (kernels.cuh:349-369) */
uint32_t orc_failure_check(const SP *p, uint32_t utility, double pp, double q)
{
    double beta, M_sq, pmin, pmax, qmax, pmin2;
    grain_params(p, &pmin, &pmax, &qmax, &beta, &M_sq, &pmin2);
    if (pp < 0) {
        if (pp < pmin2) return utility | ICEMPM_STATUS_CRUSHED;
        double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        double q_limit = k * (pp - pmin2);
        if (q > q_limit) return utility | ICEMPM_STATUS_CRUSHED;
    } else {
        double yv = (1. + 2. * beta) * q * q + M_sq * (pp + beta * pmax) * (pp - pmax);
        if (yv > 0) return utility | ICEMPM_STATUS_CRUSHED;
    }
    return utility;
}

static inline void usvt(const double U[4], const double s0, const double s1, const double V[4], double F[4])
{
    /* U * diag(s) * V^T */
    double a0 = U[0] * s0, a1 = U[1] * s1, a2 = U[2] * s0, a3 = U[3] * s1;
    F[0] = a0 * V[0] + a1 * V[1];
    F[1] = a0 * V[2] + a1 * V[3];
    F[2] = a2 * V[0] + a3 * V[1];
    F[3] = a2 * V[2] + a3 * V[3];
}

/* Wolper_Drucker_Prager (kernels.cuh:374-483).  Returns the case (0..3) and
 * sets *nan_flag when Fe became NaN. */
int orc_wolper_dp(const SP *p, double thickness, double p_tr, double q_tr, double Je_tr,
                  const double U[4], const double V[4], const double sig2[2],
                  const double shat[2], double Fe[4], double *Jp_inv, int *nan_flag)
{
    const double mu = p->mu, kappa = p->kappa;
    const double DP_threshold_p = p->DP_threshold_p;
    const double pmin = -p->IceTensileStrength;
    const double pmax = p->IceCompressiveStrength;
    const double qmax = p->IceShearStrength;
    const double tan_phi = tan(p->DP_phi * ICEMPM_PI / 180);
    int case1;
    (void)sig2;
    if (p_tr < DP_threshold_p) {
        if (*Jp_inv < 0.1) {
            case1 = 0;
            double sj = sqrt(Je_tr);
            usvt(U, sj, sj, V, Fe);
        } else {
            case1 = 1;
            usvt(U, 1.0, 1.0, V, Fe);
            *Jp_inv /= Je_tr;
        }
    } else {
        case1 = 2;
        double q_yield;
        if (p_tr < pmax) {
            double q_fs = 2 * sqrt((pmax - p_tr) * (p_tr - pmin)) * qmax / (pmax - pmin);
            double q_dp = fmax(0.0, (p_tr - DP_threshold_p) * tan_phi);
            q_yield = fmin(q_fs, q_dp);
        } else {
            q_yield = 0;
        }
        if (q_tr > q_yield) {
            case1 = 3;
            double p_ridge_max = p->RidgeFormationCoeff * ICEMPM_GRAVITY * p->IceDensity * thickness * (*Jp_inv);
            double p_n_1 = fmin(p_tr, p_ridge_max);
            double q_n_1;
            if (p_n_1 < pmax) {
                double q_dp = fmax(0.0, (p_n_1 - DP_threshold_p) * tan_phi);
                double q_fs = 2 * sqrt((pmax - p_n_1) * (p_n_1 - pmin)) * qmax / (pmax - pmin);
                q_n_1 = fmin(q_fs, q_dp);
            } else {
                q_n_1 = 0;
            }
            double Je_new = sqrt(-2 * p_n_1 / kappa + 1);
            double s_hat_n_1_norm = q_n_1 * coeff1_inv;
            double nrm2 = shat[0] * shat[0] + shat[1] * shat[1];
            double n0 = shat[0], n1 = shat[1];
            if (nrm2 > 0) { double nr = sqrt(nrm2); n0 /= nr; n1 /= nr; }
            double f = s_hat_n_1_norm * (Je_tr / mu);
            double b0 = f * n0 + Je_new;
            double b1 = f * n1 + Je_new;
            usvt(U, sqrt(b0), sqrt(b1), V, Fe);
            *Jp_inv *= Je_new / Je_tr;
        }
    }
    if (isnan(Fe[0]) || isnan(Fe[2]) || isnan(Fe[1]) || isnan(Fe[3])) *nan_flag = 1;
    return case1;
}

/* ====================================================================== */
/* P2G (kernels.cuh:39-104)                                                */
/* ====================================================================== */

/* Scatter of one point; returns error bits.  area (may be NULL) receives
 * sum(w * ParticleVolume) for the extended forcing. */
static void wind_at(const icempm_options_t *o, double x, double y, double *ux, double *uy);

static uint32_t p2g_point(const SP *p, const double *soa, size_t pitch, size_t i,
                          double *grid, size_t gpitch, size_t nnodes, const icempm_options_t *ext)
{
    uint32_t err = 0;
    const double h = p->cellsize;
    const int gridY = p->GridYTotal;
    const int gridX = p->GridXTotal;
    double pos[2], vel[2], Bp[4], Fe[4];
    for (int a = 0; a < 2; a++) {
        pos[a] = soa[i + pitch * (ICEMPM_IDX_POSX + a)];
        vel[a] = soa[i + pitch * (ICEMPM_IDX_VELX + a)];
        for (int b = 0; b < 2; b++) {
            Fe[a * 2 + b] = soa[i + pitch * (ICEMPM_IDX_FE00 + a * 2 + b)];
            Bp[a * 2 + b] = soa[i + pitch * (ICEMPM_IDX_BP00 + a * 2 + b)];
        }
    }
    const double Jp_inv = soa[i + pitch * ICEMPM_IDX_JP_INV];
    const double thickness = soa[i + pitch * ICEMPM_IDX_THICKNESS];
    const double particle_mass = p->ParticleMass * thickness;
    const uint32_t cell = slot_u32(&soa[i + pitch * ICEMPM_IDX_CELL]);
    const int cx = (int)(cell & 0xffff), cy = (int)(cell >> 16);

    double PFt[4];
    orc_kirchhoff(p, Fe, PFt);
    const double sc = p->dt_vol_Dpinv * Jp_inv * thickness;
    double sub[4];
    for (int k = 0; k < 4; k++) sub[k] = particle_mass * Bp[k] - sc * PFt[k];

    /* extended forcing: impulse of the wind and water stresses over the
       point's area during the step, distributed with the B-spline weights;
       wind and current are taken at the point's cell node */
    double fx = 0, fy = 0;
    if (ext) {
        double ux, uy;
        wind_at(ext, cx * h, cy * h, &ux, &uy);   /* wind sampled at the point's cell node */
        const double um = sqrt(ux * ux + uy * uy);
        const long long nc = (long long)cy + (long long)cx * gridY;
        double wx = 0, wy = 0;
        if (nc >= 0 && (size_t)nc < nnodes) {
            wx = grid[ICEMPM_GRID_CURRENT_VX * gpitch + nc];
            wy = grid[ICEMPM_GRID_CURRENT_VY * gpitch + nc];
        }
        const double dx = wx - vel[0], dy = wy - vel[1];
        const double dm = sqrt(dx * dx + dy * dy);
        const double ca = ext->air_density * ext->air_drag_coeff * um;
        const double cw = ext->water_density * ext->water_drag_coeff * dm;
        const double f = p->InitialTimeStep * p->ParticleVolume;
        fx = f * (ca * ux + cw * dx);
        fy = f * (ca * uy + cw * dy);
    }
    double ww[3][2];
    orc_weights(pos, ww);
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++) {
            const double Wip = ww[a + 1][0] * ww[b + 1][1];
            const double incM = Wip * particle_mass;
            const double d0 = (a - pos[0]) * h, d1 = (b - pos[1]) * h;
            double incV0 = Wip * (vel[0] * particle_mass + (sub[0] * d0 + sub[1] * d1));
            double incV1 = Wip * (vel[1] * particle_mass + (sub[2] * d0 + sub[3] * d1));
            if (ext) { incV0 += Wip * fx; incV1 += Wip * fy; }
            const long long node = (long long)(b + cy) + (long long)(a + cx) * gridY;
            if (node >= 0 && (size_t)node < nnodes) {
                grid[ICEMPM_GRID_MASS * gpitch + node] += incM;
                grid[ICEMPM_GRID_PX * gpitch + node] += incV0;
                grid[ICEMPM_GRID_PY * gpitch + node] += incV1;
            }
            if (isnan(incV0) || isnan(incV1)) err |= ICEMPM_ERR_GRID_P2G_NAN_VEL;
            if (isnan(incM)) err |= ICEMPM_ERR_GRID_P2G_NAN_MASS;
        }
    if (cx < 1 || cy < 1 || cx > (gridX - 2) || cy > gridY - 2) err |= ICEMPM_ERR_POINT_LEFT_AREA;
    return err;
}

#define ORC_STRIP 4

/* P2G over all enabled points.  Deterministic, see the file header. */
uint32_t orc_p2g(const SP *p, const double *soa, size_t pitch, size_t n,
                 double *grid, size_t gpitch, const icempm_options_t *ext)
{
    const int gx = p->GridXTotal;
    const size_t nnodes = (size_t)gx * p->GridYTotal;
    const int nstrips = (gx + ORC_STRIP - 1) / ORC_STRIP;
    size_t *start = (size_t *)calloc((size_t)nstrips + 2, sizeof(size_t));
    int32_t *sid = (int32_t *)malloc(n * sizeof(int32_t) + 1);
    size_t *order = (size_t *)malloc(n * sizeof(size_t) + 1);
    uint32_t err = 0;
    for (size_t i = 0; i < n; i++) {
        uint32_t util = slot_u32(&soa[i + pitch * ICEMPM_IDX_UTILITY]);
        if (util & ICEMPM_STATUS_DISABLED) { sid[i] = -1; continue; }
        uint32_t cell = slot_u32(&soa[i + pitch * ICEMPM_IDX_CELL]);
        int cx = (int)(cell & 0xffff);
        int s = cx / ORC_STRIP;
        if (s >= nstrips) s = nstrips - 1;
        sid[i] = s;
        start[s + 1]++;
    }
    for (int s = 0; s < nstrips; s++) start[s + 1] += start[s];
    {
        size_t *fill = (size_t *)malloc(((size_t)nstrips + 1) * sizeof(size_t));
        memcpy(fill, start, ((size_t)nstrips + 1) * sizeof(size_t));
        for (size_t i = 0; i < n; i++)
            if (sid[i] >= 0) order[fill[sid[i]]++] = i;
        free(fill);
    }
    for (int color = 0; color < 2; color++) {
        uint32_t e = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : e)
        for (int s = color; s < nstrips; s += 2)
            for (size_t k = start[s]; k < start[s + 1]; k++)
                e |= p2g_point(p, soa, pitch, order[k], grid, gpitch, nnodes, ext);
        err |= e;
    }
    free(start); free(sid); free(order);
    return err;
}

/* ====================================================================== */
/* Grid update (kernels.cuh:109-177)                                       */
/* ====================================================================== */
uint32_t orc_update_nodes(const SP *p, double *grid, size_t gpitch, const uint8_t *status,
                          double simulation_time)
{
    const long long nNodes = (long long)p->GridXTotal * p->GridYTotal;
    uint32_t err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
    for (long long idx = 0; idx < nNodes; idx++) {
        const double mass = grid[ICEMPM_GRID_MASS * gpitch + idx];
        if (mass == 0) continue;
        const double mx = grid[ICEMPM_GRID_PX * gpitch + idx];
        const double my = grid[ICEMPM_GRID_PY * gpitch + idx];
        const double vmax = p->vmax;
        double v0 = mx / mass, v1 = my / mass;
        if (status[idx] != 100) {
            v0 = 0; v1 = 0;
            grid[ICEMPM_GRID_FX * gpitch + idx] += mx;
            grid[ICEMPM_GRID_FY * gpitch + idx] += my;
        } else {
            double w0 = grid[ICEMPM_GRID_CURRENT_VX * gpitch + idx];
            double w1 = grid[ICEMPM_GRID_CURRENT_VY * gpitch + idx];
            double ramp;
            if (simulation_time < 300000) ramp = 1 + fmin(simulation_time / (3600 * 2), 2.);
            else ramp = 3 + fmin((simulation_time - 300000) / (3600 * 10), 2.);
            w0 *= ramp; w1 *= ramp;
            const double kL = p->waterDragEffectiveLinear * p->InitialTimeStep;
            const double kQp = p->waterDragEffectiveQuadratic * p->InitialTimeStep;
            const double u0 = w0 - v0, u1 = w1 - v1;
            const double umag = sqrt(u0 * u0 + u1 * u1);
            double k = kL + kQp * umag;
            k = fmin(k, 0.1);
            v0 += k * u0; v1 += k * u1;
        }
        if (v0 * v0 + v1 * v1 > vmax * vmax * 0.1) { v0 = 0; v1 = 0; }
        grid[ICEMPM_GRID_PX * gpitch + idx] = v0;
        grid[ICEMPM_GRID_PY * gpitch + idx] = v1;
        if (isnan(v0) || isnan(v1)) err |= ICEMPM_ERR_GRID_NAN;
    }
    return err;
}

/* Wind at a world position for the extended forcing (no reference counterpart). */
static void wind_at(const icempm_options_t *o, double x, double y, double *ux, double *uy)
{
    *ux = 0; *uy = 0;
    if (o->wind_kind == ICEMPM_WIND_UNIFORM) { *ux = o->wind_u; *uy = o->wind_v; }
    else if (o->wind_kind == ICEMPM_WIND_RANKINE) {
        double dx = x - o->wind_cx, dy = y - o->wind_cy;
        double r = sqrt(dx * dx + dy * dy);
        if (r > 0) {
            double sp = (r < o->wind_radius) ? o->wind_vmax * r / o->wind_radius
                                             : o->wind_vmax * o->wind_radius / r;
            *ux = -dy / r * sp; *uy = dx / r * sp;
        }
    }
}

/* Grid update of the extended forcing (no reference counterpart; the
 * reference computes a wind vector but never passes it to the kernel,
 * gpu_partition.cpp:336-348).  The wind and water stresses enter as point
 * impulses in P2G (p2g_point), so the node update is v = p/m with the
 * reference's walls and velocity clamp and neither the current ramp nor the
 * effective-coefficient drag. */
uint32_t orc_update_nodes_ext(const SP *p, double *grid, size_t gpitch, const uint8_t *status)
{
    const long long nNodes = (long long)p->GridXTotal * p->GridYTotal;
    uint32_t err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
    for (long long idx = 0; idx < nNodes; idx++) {
        const double mass = grid[ICEMPM_GRID_MASS * gpitch + idx];
        if (mass == 0) continue;
        const double mx = grid[ICEMPM_GRID_PX * gpitch + idx];
        const double my = grid[ICEMPM_GRID_PY * gpitch + idx];
        double v0 = mx / mass, v1 = my / mass;
        if (status[idx] != 100) {
            v0 = 0; v1 = 0;
            grid[ICEMPM_GRID_FX * gpitch + idx] += mx;
            grid[ICEMPM_GRID_FY * gpitch + idx] += my;
        }
        if (v0 * v0 + v1 * v1 > p->vmax * p->vmax * 0.1) { v0 = 0; v1 = 0; }
        grid[ICEMPM_GRID_PX * gpitch + idx] = v0;
        grid[ICEMPM_GRID_PY * gpitch + idx] = v1;
        if (isnan(v0) || isnan(v1)) err |= ICEMPM_ERR_GRID_NAN;
    }
    return err;
}

/* ====================================================================== */
/* G2P (kernels.cuh:181-315)                                               */
/* ====================================================================== */
uint32_t orc_g2p(const SP *p, double *soa, size_t pitch, size_t n, const double *grid,
                 size_t gpitch, int recordPQ, int32_t *disabled_count)
{
    uint32_t err = 0;
    int32_t ndis = 0;
    const double h_inv = p->cellsize_inv, dt = p->InitialTimeStep;
    const double mu = p->mu;
    const int gridY = p->GridYTotal, gridX = p->GridXTotal;
    const long long nnodes = (long long)gridX * gridY;
#pragma omp parallel for schedule(static) reduction(| : err) reduction(+ : ndis)
    for (long long ii = 0; ii < (long long)n; ii++) {
        const size_t i = (size_t)ii;
        uint32_t util = slot_u32(&soa[i + pitch * ICEMPM_IDX_UTILITY]);
        if (util & ICEMPM_STATUS_DISABLED) continue;
        double pos[2], Fe[4];
        for (int a = 0; a < 2; a++) {
            pos[a] = soa[i + pitch * (ICEMPM_IDX_POSX + a)];
            for (int b = 0; b < 2; b++) Fe[a * 2 + b] = soa[i + pitch * (ICEMPM_IDX_FE00 + a * 2 + b)];
        }
        const double thickness = soa[i + pitch * ICEMPM_IDX_THICKNESS];
        double Jp_inv = soa[i + pitch * ICEMPM_IDX_JP_INV];
        uint32_t cell = slot_u32(&soa[i + pitch * ICEMPM_IDX_CELL]);
        int cx = (int)(cell & 0xffff), cy = (int)(cell >> 16);
        double ww[3][2];
        orc_weights(pos, ww);
        double pv[2] = {0, 0}, Bp[4] = {0, 0, 0, 0};
        for (int a = -1; a <= 1; a++)
            for (int b = -1; b <= 1; b++) {
                const double dp0 = a - pos[0], dp1 = b - pos[1];
                const double weight = ww[a + 1][0] * ww[b + 1][1];
                const long long node = (long long)(b + cy) + (long long)(a + cx) * gridY;
                double nv0 = 0, nv1 = 0;
                if (node >= 0 && node < nnodes) {
                    nv0 = grid[ICEMPM_GRID_PX * gpitch + node];
                    nv1 = grid[ICEMPM_GRID_PY * gpitch + node];
                }
                pv[0] += weight * nv0;
                pv[1] += weight * nv1;
                const double cf = 4.f * h_inv * weight;
                Bp[0] += cf * (nv0 * dp0);
                Bp[1] += cf * (nv0 * dp1);
                Bp[2] += cf * (nv1 * dp0);
                Bp[3] += cf * (nv1 * dp1);
            }
        pos[0] += pv[0] * (dt * h_inv);
        pos[1] += pv[1] * (dt * h_inv);
        if (isnan(pv[0]) || isnan(pv[1])) err |= ICEMPM_ERR_POINT_VEL_NAN;
        if (isnan(pos[0]) || isnan(pos[1])) err |= ICEMPM_ERR_POINT_POS_NAN;
        if (isnan(Bp[0]) || isnan(Bp[2]) || isnan(Bp[1]) || isnan(Bp[3])) err |= ICEMPM_ERR_POINT_BP_NAN;

        int cell_updated = 0;
        if (pos[0] > 0.5) { pos[0] -= 1.0; cx++; cell_updated = 1; }
        else if (pos[0] < -0.5) { pos[0] += 1.0; cx--; cell_updated = 1; }
        if (pos[1] > 0.5) { pos[1] -= 1.0; cy++; cell_updated = 1; }
        else if (pos[1] < -0.5) { pos[1] += 1.0; cy--; cell_updated = 1; }
        if (cell_updated) {
            if (cx <= 1 || cx >= gridX - 2 || cy <= 1 || cy >= gridY - 2) {
                util |= ICEMPM_STATUS_DISABLED;
                ndis++;
            }
        }
        if (pos[0] > 0.5 || pos[0] < -0.5 || pos[1] > 0.5 || pos[1] < -0.5) err |= ICEMPM_ERR_POINT_JUMP_CELLS;

        double A[4] = {1 + dt * Bp[0], dt * Bp[1], dt * Bp[2], 1 + dt * Bp[3]};
        mul2(A, Fe, Fe);
        if (isnan(Fe[0]) || isnan(Fe[2]) || isnan(Fe[1]) || isnan(Fe[3])) err |= ICEMPM_ERR_POINT_FE_NAN;

        double Je_tr, p_tr, q_tr;
        orc_compute_pq(p, Fe, &Je_tr, &p_tr, &q_tr);
        double U[4], V[4], S[2];
        orc_svd2x2(Fe, U, S, V);
        double sig2[2] = {S[0] * S[0], S[1] * S[1]};
        double mean = (sig2[0] + sig2[1]) / 2.;
        double shat[2] = {mu / Je_tr * (sig2[0] - mean), mu / Je_tr * (sig2[1] - mean)};

        if (!(util & ICEMPM_STATUS_CRUSHED)) util = orc_failure_check(p, util, p_tr, q_tr);
        if (util & ICEMPM_STATUS_CRUSHED) {
            int nanf = 0;
            orc_wolper_dp(p, thickness, p_tr, q_tr, Je_tr, U, V, sig2, shat, Fe, &Jp_inv, &nanf);
            if (nanf) err |= ICEMPM_ERR_POINT_FE_NAN;
        }
        for (int a = 0; a < 2; a++) {
            soa[i + pitch * (ICEMPM_IDX_POSX + a)] = pos[a];
            soa[i + pitch * (ICEMPM_IDX_VELX + a)] = pv[a];
            for (int b = 0; b < 2; b++) {
                soa[i + pitch * (ICEMPM_IDX_FE00 + a * 2 + b)] = Fe[a * 2 + b];
                soa[i + pitch * (ICEMPM_IDX_BP00 + a * 2 + b)] = Bp[a * 2 + b];
            }
        }
        soa[i + pitch * ICEMPM_IDX_JP_INV] = Jp_inv;
        slot_set_u32(&soa[i + pitch * ICEMPM_IDX_UTILITY], util);
        if (cell_updated)
            slot_set_u32(&soa[i + pitch * ICEMPM_IDX_CELL], ((uint32_t)cy << 16) | (uint32_t)cx);
        if (recordPQ) {
            soa[i + pitch * ICEMPM_IDX_P] = p_tr;
            soa[i + pitch * ICEMPM_IDX_Q] = q_tr;
        }
    }
    if (disabled_count) *disabled_count += ndis;
    return err;
}

/* ====================================================================== */
/* Sub-step loop (model.cpp:18-39) on a full reference grid                */
/* ====================================================================== */
/* grid: 9 rows x gpitch doubles (current rows 5-6 and force rows 7-8 are the
 * caller's; normals are unused).  opts == NULL or forcing COMPAT runs the
 * reference update; EXTENDED runs orc_update_nodes_ext.  The simulation time
 * of step k is dt*k rounded to float, as GPU_Implementation5::update_nodes
 * takes it (gpu_implementation5.h:61, model.cpp:20-28). */
uint32_t orc_run_steps(const SP *p, const icempm_options_t *opts, double *soa, size_t pitch,
                       size_t n, double *grid, size_t gpitch, const uint8_t *status,
                       int nsteps, int first_step, int32_t *disabled_count)
{
    uint32_t err = 0;
    const size_t nn = (size_t)p->GridXTotal * p->GridYTotal;
    const icempm_options_t *ext = (opts && opts->forcing == ICEMPM_FORCING_EXTENDED) ? opts : NULL;
    (void)nn;
    for (int k = 0; k < nsteps; k++) {
        const int step = first_step + k;
        const double t = (double)(float)(p->InitialTimeStep * step);
        memset(grid, 0, 3 * gpitch * sizeof(double)); /* mass, px, py (gpu_partition.cpp:300-308) */
        err |= orc_p2g(p, soa, pitch, n, grid, gpitch, ext);
        if (ext) err |= orc_update_nodes_ext(p, grid, gpitch, status);
        else err |= orc_update_nodes(p, grid, gpitch, status, t);
        const int recordPQ = (p->UpdateEveryNthStep > 0) ? (step % p->UpdateEveryNthStep == 0) : 0;
        err |= orc_g2p(p, soa, pitch, n, grid, gpitch, recordPQ, disabled_count);
    }
    return err;
}

/* RemoveDisabledAndSort (host_side_soa.cpp:36-47): remove disabled points and
 * order the rest by x*GridY + y (stable among equal keys).  Operates in place
 * on the 19-row buffer; returns the new size. */
static int g_sort_gridY;
static const double *g_sort_soa;
static size_t g_sort_pitch;
static int cmp_key(const void *a, const void *b)
{
    size_t i = *(const size_t *)a, j = *(const size_t *)b;
    uint32_t ci = slot_u32(&g_sort_soa[i + g_sort_pitch * ICEMPM_IDX_CELL]);
    uint32_t cj = slot_u32(&g_sort_soa[j + g_sort_pitch * ICEMPM_IDX_CELL]);
    long long ki = (long long)(ci & 0xffff) * g_sort_gridY + (ci >> 16);
    long long kj = (long long)(cj & 0xffff) * g_sort_gridY + (cj >> 16);
    if (ki != kj) return ki < kj ? -1 : 1;
    return i < j ? -1 : (i > j ? 1 : 0);
}
size_t orc_remove_disabled_and_sort(double *soa, size_t pitch, size_t n, int gridY)
{
    size_t *idx = (size_t *)malloc(n * sizeof(size_t) + 1);
    size_t m = 0;
    for (size_t i = 0; i < n; i++)
        if (!(slot_u32(&soa[i + pitch * ICEMPM_IDX_UTILITY]) & ICEMPM_STATUS_DISABLED)) idx[m++] = i;
    g_sort_gridY = gridY; g_sort_soa = soa; g_sort_pitch = pitch;
    qsort(idx, m, sizeof(size_t), cmp_key);
    double *tmp = (double *)malloc((m + 1) * sizeof(double));
    for (int r = 0; r < ICEMPM_N_PTS_ARRAYS; r++) {
        for (size_t k = 0; k < m; k++) tmp[k] = soa[idx[k] + pitch * r];
        memcpy(&soa[pitch * r], tmp, m * sizeof(double));
    }
    free(tmp); free(idx);
    return m;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
