// sph_constitutive.cuh -- per-particle constitutive arithmetic of the step
// (CPP_8-1-consfactor.cpp, CPP_7-2-constitutive.cpp, Class_particle.cpp,
// CPP_7-1-strain.cpp), in the reference's operation order.
#pragma once


__device__ __forceinline__ void jaumann(double ds[6], const double s[6], const double we[9])
{
#define WE(a, b) we[(a) * 3 + (b)]
    ds[0] = ds[0] + (WE(0, 0) * s[0] + WE(0, 1) * s[3] + WE(0, 2) * s[5]) - (s[0] * WE(0, 0) + s[3] * WE(1, 0) + s[5] * WE(2, 0));
    ds[1] = ds[1] + (WE(1, 0) * s[3] + WE(1, 1) * s[1] + WE(1, 2) * s[4]) - (s[3] * WE(0, 1) + s[1] * WE(1, 1) + s[4] * WE(2, 1));
    ds[2] = ds[2] + (WE(2, 0) * s[5] + WE(2, 1) * s[4] + WE(2, 2) * s[2]) - (s[5] * WE(0, 2) + s[4] * WE(1, 2) + s[2] * WE(2, 2));
    ds[3] = ds[3] + (WE(0, 0) * s[3] + WE(0, 1) * s[1] + WE(0, 2) * s[4]) - (s[0] * WE(0, 1) + s[3] * WE(1, 1) + s[5] * WE(2, 1));
    ds[4] = ds[4] + (WE(1, 0) * s[5] + WE(1, 1) * s[4] + WE(1, 2) * s[2]) - (s[3] * WE(0, 2) + s[1] * WE(1, 2) + s[4] * WE(2, 2));
    ds[5] = ds[5] + (WE(0, 0) * s[5] + WE(0, 1) * s[4] + WE(0, 2) * s[2]) - (s[0] * WE(0, 2) + s[3] * WE(1, 2) + s[5] * WE(2, 2));
#undef WE
}

// elastic D (only its nonzero pattern is kept: dlam, dmu) -- elastic(),
// dpmodel1(), dpmodel_bui() share it (:17-59, :301-334, :468-501)
// (elastic_plastic, :618-660, takes the mean stress with third = 0.333333333)
// The elastic modulus: the material's E, or 3 (1 - 2 nu) (1 + e0) |p| / kappa
// when E <= 1 (p = mean compression, at least 1).
__device__ __forceinline__ double elastic_e0(const double s[6], double E, double poi, double eps0, double kapa,
                                             double* sm_out, double third = 0.3333333333)
{
    double sm = (-s[0] + -s[1] + -s[2]) * third;
    if (sm < 1.0) sm = 1.0;
    double e0;
    if (E > 1.0) e0 = E;
    else e0 = 3 * (1 - 2 * poi) * (1 + eps0) * fabs(sm) / kapa;
    *sm_out = sm;
    return e0;
}

__device__ __forceinline__ void elastic_consts(const double s[6], double E, double poi, double eps0, double kapa,
                                               double* dlam, double* dmu, double* sm_out,
                                               double third = 0.3333333333)
{
    double sm;
    const double e0 = elastic_e0(s, E, poi, eps0, kapa, &sm, third);
    *dlam = e0 * poi / (1.0 + poi) / (1.0 - 2.0 * poi);
    *dmu = e0 * 0.5 / (1.0 + poi);
    *sm_out = sm;
}

// dsig += D deps, in the reference's dept[ki][kj] * deps[kj] loop order over a
// dense 6x6 with the zero entries included (0 * x terms keep signed-zero and
// NaN behaviour identical).
__device__ __forceinline__ void add_dense(double ds[6], const double D[6][6], const double de[6])
{
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) ds[a] += D[a][b] * de[b];
}

__device__ __forceinline__ void fill_elastic(double D[6][6], double dlam, double dmu)
{
    const double dmu2 = dmu * 2.0;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) D[a][b] = 0.0;
    D[0][0] = dlam + dmu2; D[1][1] = dlam + dmu2; D[2][2] = dlam + dmu2;
    D[0][1] = dlam; D[0][2] = dlam; D[1][0] = dlam;
    D[1][2] = dlam; D[2][0] = dlam; D[2][1] = dlam;
    D[3][3] = dmu; D[4][4] = dmu; D[5][5] = dmu;
}

// Drucker-Prager continuum tangent (dpmodel1 / dpmodel_bui, :284-448 /
// :451-615) and, with MC = true, the Mohr-Coulomb form of elastic_plastic
// (:618-777: plastic potential without dilatancy and no hardening term in
// the denominator).  yalf, ykap, yalf_dil are the material constants the
// reference evaluates with atan/tan/sin/cos each call; they are evaluated once
// per particle by the host with the same libm calls.
template <bool MC = false>
__device__ __forceinline__ void dp_tangent(double D[6][6], double adps[6], const double s[6], const double de[6],
                                           double dlam, double dmu, double sm,
                                           double yalf, double ykap, double yalf_dil)
{
    const double dmu2 = dmu * 2.0;
    double sig0 = -s[0], sig1 = -s[1], sig2 = -s[2];
    double dx = sig0 - sm, dy = sig1 - sm, dz = sig2 - sm;
    double dxy = -s[3], dyz = -s[4], dzx = -s[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double sj = sqrt(sjj);
    if ((sj - yalf * sm * 3.0 - ykap) >= 0.0) {
        double f11 = -yalf + dx / sj * 0.5, f22 = -yalf + dy / sj * 0.5, f33 = -yalf + dz / sj * 0.5;
        double f12 = dxy / sj * 0.5, f23 = dyz / sj * 0.5, f31 = dzx / sj * 0.5;
        double fkk = f11 + f22 + f33;
        double g11 = MC ? dx / sj * 0.5 : -yalf_dil + dx / sj * 0.5;
        double g22 = MC ? dy / sj * 0.5 : -yalf_dil + dy / sj * 0.5;
        double g33 = MC ? dz / sj * 0.5 : -yalf_dil + dz / sj * 0.5;
        double g12 = dxy / sj * 0.5, g23 = dyz / sj * 0.5, g31 = dzx / sj * 0.5;
        double hdd = g11 + g22 + g33;
        double fij = 2.0 * (f11 * g11 + f22 * g22 + f33 * g33) + f12 * g12 + f23 * g23 + f31 * g31;
        double cc7 = MC ? dlam * (fkk * hdd) + dmu * fij : dlam * (fkk * hdd) + dmu * fij + hdd;
        double dd_ = 1.0 / cc7;
        double df = dlam * fkk, dg = dlam * hdd;
        double ramda = (dmu2 * f11 - 3.0 * dlam * yalf) * de[0]
            + (dmu2 * f22 - 3.0 * dlam * yalf) * de[1]
            + (dmu2 * f33 - 3.0 * dlam * yalf) * de[2]
            + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
        double ttt = ramda * dd_;
        if (ttt < 0.0) {
            double ww[6] = {dg + dmu2 * g11, dg + dmu2 * g22, dg + dmu2 * g33, dmu * g12, dmu * g23, dmu * g31};
            double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
            for (int a = 0; a < 6; a++)
                for (int b = 0; b < 6; b++) D[a][b] = D[a][b] - dd_ * ww[a] * zz[b];
            adps[0] = ramda * dd_ * f11; adps[1] = ramda * dd_ * f22; adps[2] = ramda * dd_ * f33;
            adps[3] = ramda * dd_ * f12; adps[4] = ramda * dd_ * f23; adps[5] = ramda * dd_ * f31;
        }
    }
}

// sub_camclay: subloading Cam-clay tangent (:129-281).  ymf from the
// critical-state ratio zmf; the subloading ratio term roue from log(sme0 / sm).
__device__ __forceinline__ void subcam_tangent(double D[6][6], double adps[6], const double s[6], const double de[6],
                                               double dlam, double dmu, double sm, double ann, double zmf,
                                               double zramda, double zkapa, double eps0, double sme0, double fs)
{
    const double dmu2 = dmu * 2.0;
    const double ymf = 3.0 * (zmf - 1.0) / (zmf + 2.0) / fs;
    const double hee = (zramda - zkapa) / (1.0 + eps0);
    double dx = -s[0] - sm, dy = -s[1] - sm, dz = -s[2] - sm;
    double dxy = -s[3], dyz = -s[4], dzx = -s[5];
    double sjj = 0.5 * (dx * dx + dy * dy + dz * dz) + dxy * dxy + dyz * dyz + dzx * dzx;
    double tt1 = 1.0 / (ymf * ymf * sm * sm + 3.0 * sjj);
    double tt2 = 2.0 * ymf * ymf * sm * tt1 - 1.0 / sm;
    double f11 = tt2 / 3.0 + dx * tt1 * 3.0;
    double f22 = tt2 / 3.0 + dy * tt1 * 3.0;
    double f33 = tt2 / 3.0 + dz * tt1 * 3.0;
    double f12 = 3.0 * dxy * tt1, f23 = 3.0 * dyz * tt1, f31 = 3.0 * dzx * tt1;
    double roue = (1 + eps0) * log(sme0 / sm);
    if (roue < 0.0) roue = 0.0;
    double ttt = ann * roue * roue;
    double hdd = f11 + f22 + f33 + ttt / sm;
    double fkk = f11 + f22 + f33;
    double fij = 2.0 * (f11 * f11 + f22 * f22 + f33 * f33) + f12 * f12 + f23 * f23 + f31 * f31;
    double cc7 = dlam * (fkk * fkk) + dmu * fij + hdd / hee;
    double dd_ = 1.0 / cc7;
    double df = dlam * fkk, dg = dlam * fkk;
    double ramda = (dmu2 * f11 + dlam * fkk) * de[0] + (dmu2 * f22 + dlam * fkk) * de[1]
        + (dmu2 * f33 + dlam * fkk) * de[2] + dmu * (f12 * de[3] + f23 * de[4] + f31 * de[5]);
    if (ramda < 0.0) {
        double ww[6] = {dg + dmu2 * f11, dg + dmu2 * f22, dg + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        double zz[6] = {df + dmu2 * f11, df + dmu2 * f22, df + dmu2 * f33, dmu * f12, dmu * f23, dmu * f31};
        for (int a = 0; a < 6; a++)
            for (int b = 0; b < 6; b++) D[a][b] = D[a][b] - dd_ * ww[a] * zz[b];
        adps[0] = ramda * dd_ * f11; adps[1] = ramda * dd_ * f22; adps[2] = ramda * dd_ * f33;
        adps[3] = ramda * dd_ * f12; adps[4] = ramda * dd_ * f23; adps[5] = ramda * dd_ * f31;
    }
}

// viscous_elastic (:88-126): dsig set directly, bulk modulus from the
// elastic modulus, shear modulus g = the material's c
__device__ __forceinline__ void visco_elastic(double ds[6], const double de[6], double e0, double poi, double g)
{
    const double k = e0 * 0.3333333333 / (1.0 - 2.0 * poi);
    const double epkk = de[0] + de[1] + de[2];
    ds[0] = 2.0 * g * (de[0] - epkk * 0.3333333333) + k * epkk;
    ds[1] = 2.0 * g * (de[1] - epkk * 0.3333333333) + k * epkk;
    ds[2] = 2.0 * g * (de[2] - epkk * 0.3333333333) + k * epkk;
    ds[3] = 2.0 * g * de[3];
    ds[4] = 2.0 * g * de[4];
    ds[5] = 2.0 * g * de[5];
}

// DPModel_check: stress-scaling return onto the cone (:779-819)
__device__ __forceinline__ void dp_check(const double s[6], double ds[6], double alpha_fai, double k_c, double dt)
{
    double ts[6];
    double sm = (s[0] + s[1] + s[2]) / 3.0;
    double dx = s[0] - sm, dy = s[1] - sm, dz = s[2] - sm;
    double sj_2 = 0.5 * (dx * dx + dy * dy + dz * dz) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    double sj = sqrt(sj_2);
    for (int a = 0; a < 6; a++) ts[a] = s[a] + ds[a] * dt;
    double i_1 = ts[0] + ts[1] + ts[2];
    double rn = (-alpha_fai * i_1 + k_c) / sj;
    if (rn < 1.0) {
        ts[0] = rn * (ts[0] - i_1 / 3.0) + i_1 / 3.0;
        ts[1] = rn * (ts[1] - i_1 / 3.0) + i_1 / 3.0;
        ts[2] = rn * (ts[2] - i_1 / 3.0) + i_1 / 3.0;
        ts[3] = rn * ts[3];
        ts[4] = rn * ts[4];
        ts[5] = rn * ts[5];
    }
    for (int a = 0; a < 6; a++) ds[a] = (ts[a] - s[a]) / dt;
}

// Particle::deq (Class_particle.cpp:121-143): vsig, veps, divq, divr
__device__ __forceinline__ void deq(const double s[6], const double ep[6], double* vsig, double* veps,
                                    double* divq, double* divr)
{
    *veps = ep[0] + ep[1] + ep[2];
    double vs = (s[0] + s[1] + s[2]) / 3;
    double sxx = s[0] - vs, syy = s[1] - vs, szz = s[2] - vs;
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5];
    double q = sqrt(3 * fabs(j2));
    *vsig = vs;
    *divq = q;
    *divr = (vs != 0.0) ? fabs(q / vs) : 0.0;
}

// Particle::shearstrain (Class_particle.cpp:175-192)
__device__ __forceinline__ double shearstrain(const double ep[6], double veps)
{
    double sxx = ep[0] - veps / 3.0, syy = ep[1] - veps / 3.0, szz = ep[2] - veps / 3.0;
    double j2 = 0.5 * (sxx * sxx + syy * syy + szz * szz) + ep[3] * ep[3] + ep[4] * ep[4] + ep[5] * ep[5];
    return sqrt(2.0 * fabs(j2));
}

// eejcb with its eigenvector matrix v (row-major, v[i*3+j]), as
// Stress_eigValue uses it for beta / beta_ts (CPP_7-1-strain.cpp:311-330,
// 341-437).
__device__ __forceinline__ void eig3v(const double s[6], double strep[3], double v[9])
{
    double a[9] = {s[0], s[3], s[5], s[3], s[1], s[4], s[5], s[4], s[2]};
    const int n = 3;
    for (int i = 0; i < 9; i++) v[i] = (i % 4 == 0) ? 1.0 : 0.0;
    int p = 0, q = 0, l = 1;
    while (true) {
        double fm = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double dd_ = fabs(a[i * n + j]);
                if ((i != j) && (dd_ > fm)) { fm = dd_; p = i; q = j; }
            }
        if (fm < 0.001) break;
        if (l > 7) break;
        l = l + 1;
        int u = p * n + q, w = p * n + p, t = q * n + p, sidx = q * n + q;
        double x = -a[u];
        double y = (a[sidx] - a[w]) / 2.0;
        double omega = x / sqrt(x * x + y * y);
        if (y < 0.0) omega = -omega;
        double sn = 1.0 + sqrt(1.0 - omega * omega);
        sn = omega / sqrt(2.0 * sn);
        double cn = sqrt(1.0 - sn * sn);
        fm = a[w];
        a[w] = fm * cn * cn + a[sidx] * sn * sn + a[u] * omega;
        a[sidx] = fm * sn * sn + a[sidx] * cn * cn - a[u] * omega;
        a[u] = 0.0;
        a[t] = 0.0;
        for (int j = 0; j < n; j++)
            if ((j != p) && (j != q)) {
                int uu = p * n + j, ww = q * n + j;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++)
            if ((i != p) && (i != q)) {
                int uu = i * n + p, ww = i * n + q;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++) {
            int uu = i * n + p, ww = i * n + q;
            fm = v[uu];
            v[uu] = fm * cn + v[ww] * sn;
            v[ww] = -fm * sn + v[ww] * cn;
        }
    }
    strep[0] = a[0]; strep[1] = a[4]; strep[2] = a[8];
}

// inverse_mat of the artificial stress (CPP_9-5-artificialstress.cpp:297-317):
// B is left unchanged (zero) when |det| <= 1e-5
__device__ __forceinline__ void inv3_or_keep(const double A[9], double B[9])
{
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[3] * (A[1] * A[8] - A[2] * A[7])
        + A[6] * (A[1] * A[5] - A[2] * A[4]);
    if (fabs(det) > 1.0e-5) {
        B[0] = (A[4] * A[8] - A[5] * A[7]) / det;
        B[1] = (A[2] * A[7] - A[1] * A[8]) / det;
        B[2] = (A[1] * A[5] - A[2] * A[4]) / det;
        B[3] = (A[5] * A[6] - A[3] * A[8]) / det;
        B[4] = (A[0] * A[8] - A[2] * A[6]) / det;
        B[5] = (A[3] * A[2] - A[0] * A[5]) / det;
        B[6] = (A[3] * A[7] - A[4] * A[6]) / det;
        B[7] = (A[1] * A[6] - A[0] * A[7]) / det;
        B[8] = (A[0] * A[4] - A[3] * A[1]) / det;
    }
}

// matrix_multiply (CPP_9-5-artificialstress.cpp:13-26), row-major 3x3
__device__ __forceinline__ void mul3(const double a[9], const double b[9], double c[9])
{
    for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) c[r * 3 + q] = a[r * 3] * b[q] + a[r * 3 + 1] * b[3 + q] + a[r * 3 + 2] * b[6 + q];
}

// eejcb Jacobi rotations, eps = 1e-3, at most 7 (CPP_7-1-strain.cpp:341-437);
// returns the diagonal (principal stresses strep).
__device__ __forceinline__ void eig3(const double s[6], double strep[3])
{
    double a[9] = {s[0], s[3], s[5], s[3], s[1], s[4], s[5], s[4], s[2]};
    const int n = 3;
    int p = 0, q = 0, l = 1;
    while (true) {
        double fm = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++) {
                double dd_ = fabs(a[i * n + j]);
                if ((i != j) && (dd_ > fm)) { fm = dd_; p = i; q = j; }
            }
        if (fm < 0.001) break;
        if (l > 7) break;
        l = l + 1;
        int u = p * n + q, w = p * n + p, t = q * n + p, sidx = q * n + q;
        double x = -a[u];
        double y = (a[sidx] - a[w]) / 2.0;
        double omega = x / sqrt(x * x + y * y);
        if (y < 0.0) omega = -omega;
        double sn = 1.0 + sqrt(1.0 - omega * omega);
        sn = omega / sqrt(2.0 * sn);
        double cn = sqrt(1.0 - sn * sn);
        fm = a[w];
        a[w] = fm * cn * cn + a[sidx] * sn * sn + a[u] * omega;
        a[sidx] = fm * sn * sn + a[sidx] * cn * cn - a[u] * omega;
        a[u] = 0.0;
        a[t] = 0.0;
        for (int j = 0; j < n; j++)
            if ((j != p) && (j != q)) {
                int uu = p * n + j, ww = q * n + j;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
        for (int i = 0; i < n; i++)
            if ((i != p) && (i != q)) {
                int uu = i * n + p, ww = i * n + q;
                fm = a[uu];
                a[uu] = fm * cn + a[ww] * sn;
                a[ww] = -fm * sn + a[ww] * cn;
            }
    }
    strep[0] = a[0]; strep[1] = a[4]; strep[2] = a[8];
}
