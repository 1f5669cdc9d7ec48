/*
 * nnp_oracle.c -- plain-C restatement of n2p2's short-range (2G) HDNNP
 * energy/force evaluation, used ONLY as test infrastructure (the checker of
 * the CUDA path and the "port" CPU baseline).  The product never links it.
 *
 * It restates, per structure and in FP64 with no FMA contraction
 * (-ffp-contract=off), the algorithm of the reference:
 *   remap                Structure::remap            Structure.cpp:1224-1248
 *   periodic copies      Structure::calculatePbcCopies Structure.cpp:485-516
 *   neighbour list       Structure::calculateNeighborList Structure.cpp:287-398
 *   cutoff functions     CutoffFunction::fdf          CutoffFunction.h:210-220,
 *                        CutoffFunction.cpp:95-213, CoreFunction.h:239-318
 *   G2 / G3 / G9 with dG/dr, one symmetry function at a time, as the
 *                        reference's ungrouped path  SymFncExpRad.cpp:111-160,
 *                        SymFncExpAngn.cpp:79-225, SymFncExpAngw.cpp:79-220
 *   scaling              SymFnc::scale               SymFnc.cpp:169-195
 *   atomic networks      NeuralNetwork::propagateLayer NeuralNetwork.cpp:761-896
 *                        and calculateDEdG            NeuralNetwork.cpp:396-442
 *   energy / forces      Mode::calculateEnergy / calculateForces
 *                        Mode.cpp:1876-1984, Atom.cpp:371-401
 * The set-up (settings parsing, symmetry-function order, scaling and weight
 * files) is done by oracle/port.py and handed over as flat arrays.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
    int numElements;
    double maxCutoff;
    int cutoffType;
    double cutoffAlpha;
    /* symmetry functions, all elements concatenated in sorted order */
    int totalSF;
    const int* sfBegin;      /* [numElements+1] */
    const int* type;         /* 2, 3, 9 */
    const int* e1;
    const int* e2;
    const double* eta;
    const double* rs;
    const double* lambda;
    const double* zeta;
    const double* rc;
    const int* row;          /* [totalSF][numElements] derivative row or -1 */
    const int* numRows;      /* [numElements][numElements] */
    const int* rowSF;        /* [numElements][numElements][maxRows]: SF index (within element) of each row */
    int maxRows;
    /* scaling per SF */
    const int* scalingType;
    const double* Smin;
    const double* Gmin;
    const double* Gmax;
    const double* Gmean;
    const double* scalingFactor;
    /* networks */
    const int* numLayers;    /* [numElements] */
    const int* neurons;      /* [numElements][8] */
    const int* activation;   /* [numElements][8] */
    const int* wBegin;       /* [numElements][8] offset of layer l weights (l >= 1) */
    const int* bBegin;       /* [numElements][8] */
    const double* weights;
    int normalizeNeurons;
    /* units */
    int normalize;
    double meanEnergy, convEnergy, convLength;
    const double* atomicEnergyOffset; /* [numElements] */
} OracleModel;

typedef struct
{
    int numAtoms;
    double energy;            /* physical units, offsets added */
    double energyInternal;
    double* forces;           /* [N][3] physical */
    double* positions;        /* [N][3] internal (remapped, normalised) */
    int64_t* nbrOffset;       /* [N+1] */
    int64_t* nbrIndex;
    double* nbrD;
    double* nbrDr;            /* [M][3] */
    int64_t* sfOffset;        /* [N+1] */
    double* G;
    double* dEdG;
    double* atomicEnergy;
    int64_t warnings;
} OracleResult;

/* ----------------------------------------------------------------------- */

static void cutoff_fdf(int type, double alpha, double rc, double r, double* fc, double* dfc)
{
    const double PI = 4.0 * atan(1.0);
    const double E = exp(1.0);
    if (r >= rc)
    {
        *fc = 0.0;
        *dfc = 0.0;
        return;
    }
    double rcinv = 1.0 / rc;
    double rci = rc * alpha;
    double iw = 1.0 / (rc - rci);
    if (type == 0)
    {
        *fc = 1.0;
        *dfc = 0.0;
        return;
    }
    if (type == 2 || type == 3)
    {
        double pre = 1.0;
        if (type == 3) pre = pow((E + 1 / E) / (E - 1 / E), 3);
        double t = tanh(1.0 - r * rcinv);
        double t2 = t * t;
        *fc = pre * t * t2;
        *dfc = 3.0 * pre * t2 * (t2 - 1.0) * rcinv;
        return;
    }
    if (r < rci)
    {
        *fc = 1.0;
        *dfc = 0.0;
        return;
    }
    double x = (r - rci) * iw;
    if (type == 1)
    {
        double c = cos(PI * x);
        *fc = 0.5 * (c + 1.0);
        *dfc = -0.5 * iw * PI * sqrt(1.0 - c * c);
        return;
    }
    double f, df;
    if (type == 4)
    {
        double t = 1.0 / (x * x - 1.0);
        double e = exp(t);
        f = E * e;
        df = -2.0 * E * x * t * t * e;
    }
    else if (type == 5)
    {
        f = (2.0 * x - 3.0) * x * x + 1.0;
        df = x * (6.0 * x - 6.0);
    }
    else if (type == 6)
    {
        double x2 = x * x;
        f = ((15.0 - 6.0 * x) * x - 10.0) * x * x2 + 1.0;
        df = x2 * ((60.0 - 30.0 * x) * x - 30.0);
    }
    else if (type == 7)
    {
        double x2 = x * x;
        f = (x * (x * (20.0 * x - 70.0) + 84.0) - 35.0) * x2 * x2 + 1.0;
        df = x2 * x * (x * (x * (140.0 * x - 420.0) + 420.0) - 140.0);
    }
    else
    {
        double x4 = x * x;
        x4 *= x4;
        f = (x * (x * ((315.0 - 70.0 * x) * x - 540.0) + 420.0) - 126.0) * x * x4 + 1.0;
        df = x4 * (x * (x * ((2520.0 - 630.0 * x) * x - 3780.0) + 2520.0) - 630.0);
    }
    *fc = f;
    *dfc = df * iw;
}

/* Cutoff function value and derivative (exported for the known-answer test). */
void oracle_cutoff(int type, double alpha, double rc, double r, double* fc, double* dfc)
{
    cutoff_fdf(type, alpha, rc, r, fc, dfc);
}

/* exponentiation by squaring (the algorithm of utility.cpp:292-316) */
static double pow_by_squaring(double x, int n)
{
    unsigned m;
    if (n < 0)
    {
        x = 1.0 / x;
        m = (unsigned)(-n);
    }
    else m = (unsigned)n;
    double r = 1.0;
    do
    {
        if (m & 1u) r *= x;
        m >>= 1;
        x *= x;
    } while (m);
    return r;
}

static double scale_value(const OracleModel* M, int s, double v)
{
    switch (M->scalingType[s])
    {
    case 0: return v;
    case 1: return M->Smin[s] + M->scalingFactor[s] * (v - M->Gmin[s]);
    case 2: return v - M->Gmean[s];
    case 3:
    case 4: return M->Smin[s] + M->scalingFactor[s] * (v - M->Gmean[s]);
    }
    return 0.0;
}

static double unscale_value(const OracleModel* M, int s, double v)
{
    switch (M->scalingType[s])
    {
    case 0: return v;
    case 1: return (v - M->Smin[s]) / M->scalingFactor[s] + M->Gmin[s];
    case 2: return v + M->Gmean[s];
    case 3:
    case 4: return (v - M->Smin[s]) / M->scalingFactor[s] + M->Gmean[s];
    }
    return 0.0;
}

static void activation(int a, double x, double* y, double* dy)
{
    const double LIM = 35.0;
    switch (a)
    {
    case 1: *y = x; *dy = 1.0; return;
    case 2: { double t = tanh(x); *y = t; *dy = 1.0 - t * t; return; }
    case 3:
        if (x > LIM) { *y = 1.0; *dy = 0.0; }
        else if (x < -LIM) { *y = 0.0; *dy = 0.0; }
        else { double t = 1.0 / (1.0 + exp(-x)); *y = t; *dy = t * (1.0 - t); }
        return;
    case 4:
        if (x > LIM) { *y = x; *dy = 1.0; }
        else if (x < -LIM) { *y = 0.0; *dy = 0.0; }
        else { double t = exp(x); *y = log(1.0 + t); *dy = 1.0 / (1.0 + 1.0 / t); }
        return;
    case 5: if (x > 0.0) { *y = x; *dy = 1.0; } else { *y = 0.0; *dy = 0.0; } return;
    case 6: { double t = exp(-0.5 * x * x); *y = t; *dy = -x * t; return; }
    case 7: *y = cos(x); *dy = -sin(x); return;
    case 8: { double t = 1.0 / (1.0 + exp(-x)); *y = 1.0 - t; *dy = t * (t - 1.0); return; }
    case 9: { double t = exp(-x); *y = t; *dy = -t; return; }
    case 10: *y = x * x; *dy = 2.0 * x; return;
    }
    *y = 0.0;
    *dy = 0.0;
}

/* ----------------------------------------------------------------------- */

static void inverse_box(const double* b, double* ib)
{
#define B(k, c) b[(k) * 3 + (c)]
    double det = B(0, 0) * B(1, 1) * B(2, 2) + B(1, 0) * B(2, 1) * B(0, 2) + B(2, 0) * B(0, 1) * B(1, 2) -
                 B(2, 0) * B(1, 1) * B(0, 2) - B(0, 0) * B(2, 1) * B(1, 2) - B(1, 0) * B(0, 1) * B(2, 2);
    double inv = 1.0 / det;
    ib[0] = B(1, 1) * B(2, 2) - B(2, 1) * B(1, 2);
    ib[1] = B(2, 1) * B(0, 2) - B(0, 1) * B(2, 2);
    ib[2] = B(0, 1) * B(1, 2) - B(1, 1) * B(0, 2);
    ib[3] = B(2, 0) * B(1, 2) - B(1, 0) * B(2, 2);
    ib[4] = B(0, 0) * B(2, 2) - B(2, 0) * B(0, 2);
    ib[5] = B(1, 0) * B(0, 2) - B(0, 0) * B(1, 2);
    ib[6] = B(1, 0) * B(2, 1) - B(2, 0) * B(1, 1);
    ib[7] = B(2, 0) * B(0, 1) - B(0, 0) * B(2, 1);
    ib[8] = B(0, 0) * B(1, 1) - B(1, 0) * B(0, 1);
    for (int k = 0; k < 9; ++k) ib[k] *= inv;
#undef B
}

static void cross3(const double* a, const double* v, double* w)
{
    w[0] = a[1] * v[2] - a[2] * v[1];
    w[1] = a[2] * v[0] - a[0] * v[2];
    w[2] = a[0] * v[1] - a[1] * v[0];
}

static void unit3(double* v)
{
    double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= n;
    v[1] /= n;
    v[2] /= n;
}

typedef struct
{
    int j;
    double d;
    double dr[3];
    double* dGdr;   /* numRows[ec][ej] * 3 */
} Nbr;

void oracle_free_result(OracleResult* R)
{
    free(R->forces);
    free(R->positions);
    free(R->nbrOffset);
    free(R->nbrIndex);
    free(R->nbrD);
    free(R->nbrDr);
    free(R->sfOffset);
    free(R->G);
    free(R->dEdG);
    free(R->atomicEnergy);
    memset(R, 0, sizeof(*R));
}

/*
 * Evaluate one structure.  rIn: physical positions [N][3]; box: physical
 * [3][3] (NULL for a cluster).  Returns 0 on success.
 */
int oracle_evaluate(const OracleModel* M, int N, const double* rIn, const int* elem, const double* boxIn,
                    int useForces, OracleResult* R)
{
    memset(R, 0, sizeof(*R));
    R->numAtoms = N;
    const int NE = M->numElements;
    double box[9] = {0}, ib[9] = {0};
    double* r = (double*)malloc(sizeof(double) * 3 * N);
    memcpy(r, rIn, sizeof(double) * 3 * N);
    int periodic = boxIn != NULL;
    /* remap into the cell in physical units */
    if (periodic)
    {
        memcpy(box, boxIn, sizeof(box));
        inverse_box(box, ib);
        for (int a = 0; a < N; ++a)
        {
            double f[3], x[3] = {r[3 * a], r[3 * a + 1], r[3 * a + 2]};
            for (int c = 0; c < 3; ++c)
            {
                double t = x[0] * ib[0 * 3 + c];
                t = t + x[1] * ib[1 * 3 + c];
                t = t + x[2] * ib[2 * 3 + c];
                f[c] = t;
            }
            for (int c = 0; c < 3; ++c)
            {
                if (f[c] > 1.0) f[c] -= (int)f[c];
                if (f[c] < 0.0) f[c] += 1.0 - (int)f[c];
                if (f[c] == 1.0) f[c] = 0.0;
            }
            for (int c = 0; c < 3; ++c)
            {
                double t = f[0] * box[0 * 3 + c];
                t = t + f[1] * box[1 * 3 + c];
                t = t + f[2] * box[2 * 3 + c];
                r[3 * a + c] = t;
            }
        }
    }
    if (M->normalize)
    {
        for (int q = 0; q < 3 * N; ++q) r[q] *= M->convLength;
        for (int q = 0; q < 9; ++q) box[q] *= M->convLength;
    }
    R->positions = r;
    const double rc = M->maxCutoff;
    const double rc2 = rc * rc;
    int pbc[3] = {0, 0, 0};
    if (periodic)
    {
        double axb[3], axc[3], bxc[3], proj[3];
        cross3(box + 0, box + 3, axb);
        unit3(axb);
        cross3(box + 0, box + 6, axc);
        unit3(axc);
        cross3(box + 3, box + 6, bxc);
        unit3(bxc);
        proj[0] = fabs(box[0] * bxc[0] + box[1] * bxc[1] + box[2] * bxc[2]);
        proj[1] = fabs(box[3] * axc[0] + box[4] * axc[1] + box[5] * axc[2]);
        proj[2] = fabs(box[6] * axb[0] + box[7] * axb[1] + box[8] * axb[2]);
        for (int a = 0; a < 3; ++a)
            while (pbc[a] * proj[a] <= rc) pbc[a]++;
    }
    /* neighbour lists: j ascending, images in (bc0, bc1, bc2) order */
    int64_t cap = 1024, M_ = 0;
    Nbr* nb = (Nbr*)malloc(sizeof(Nbr) * cap);
    int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (N + 1));
    off[0] = 0;
    for (int i = 0; i < N; ++i)
    {
        for (int j = 0; j < N; ++j)
        {
            for (int b0 = -pbc[0]; b0 <= pbc[0]; ++b0)
                for (int b1 = -pbc[1]; b1 <= pbc[1]; ++b1)
                    for (int b2 = -pbc[2]; b2 <= pbc[2]; ++b2)
                    {
                        if (i == j && b0 == 0 && b1 == 0 && b2 == 0) continue;
                        if (!periodic && i == j) continue;
                        double dr[3];
                        for (int c = 0; c < 3; ++c)
                        {
                            double v = r[3 * i + c] - r[3 * j + c];
                            v = v + box[0 * 3 + c] * b0;
                            v = v + box[1 * 3 + c] * b1;
                            v = v + box[2 * 3 + c] * b2;
                            dr[c] = v;
                        }
                        double n2 = dr[0] * dr[0] + dr[1] * dr[1];
                        n2 = n2 + dr[2] * dr[2];
                        if (n2 <= rc2)
                        {
                            if (M_ == cap)
                            {
                                cap *= 2;
                                nb = (Nbr*)realloc(nb, sizeof(Nbr) * cap);
                            }
                            nb[M_].j = j;
                            nb[M_].d = sqrt(n2);
                            memcpy(nb[M_].dr, dr, sizeof(dr));
                            nb[M_].dGdr = NULL;
                            M_++;
                        }
                    }
        }
        off[i + 1] = M_;
    }
    R->nbrOffset = off;
    R->nbrIndex = (int64_t*)malloc(sizeof(int64_t) * (M_ > 0 ? M_ : 1));
    R->nbrD = (double*)malloc(sizeof(double) * (M_ > 0 ? M_ : 1));
    R->nbrDr = (double*)malloc(sizeof(double) * 3 * (M_ > 0 ? M_ : 1));
    for (int64_t e = 0; e < M_; ++e)
    {
        R->nbrIndex[e] = nb[e].j;
        R->nbrD[e] = nb[e].d;
        memcpy(R->nbrDr + 3 * e, nb[e].dr, sizeof(double) * 3);
    }
    /* symmetry functions with derivatives */
    R->sfOffset = (int64_t*)malloc(sizeof(int64_t) * (N + 1));
    R->sfOffset[0] = 0;
    for (int i = 0; i < N; ++i)
    {
        int ec = elem[i];
        R->sfOffset[i + 1] = R->sfOffset[i] + (M->sfBegin[ec + 1] - M->sfBegin[ec]);
    }
    int64_t totalG = R->sfOffset[N];
    R->G = (double*)calloc(totalG > 0 ? totalG : 1, sizeof(double));
    R->dEdG = (double*)calloc(totalG > 0 ? totalG : 1, sizeof(double));
    double* dGself = (double*)calloc(3 * (totalG > 0 ? totalG : 1), sizeof(double));
    for (int64_t e = 0; e < M_; ++e) nb[e].dGdr = NULL;
    for (int i = 0; i < N; ++i)
    {
        int ec = elem[i];
        for (int64_t e = off[i]; e < off[i + 1]; ++e)
            nb[e].dGdr = (double*)calloc(3 * (M->numRows[ec * NE + elem[nb[e].j]] + 1), sizeof(double));
        for (int s = M->sfBegin[ec]; s < M->sfBegin[ec + 1]; ++s)
        {
            int si = s - M->sfBegin[ec];
            double* gs = dGself + 3 * (R->sfOffset[i] + si);
            double sum = 0.0;
            double rcs = M->rc[s];
            if (M->type[s] == 2)
            {
                for (int64_t e = off[i]; e < off[i + 1]; ++e)
                {
                    Nbr* n = &nb[e];
                    if (elem[n->j] != M->e1[s] || !(n->d < rcs)) continue;
                    double fc, dfc;
                    cutoff_fdf(M->cutoffType, M->cutoffAlpha, rcs, n->d, &fc, &dfc);
                    double x = n->d - M->rs[s];
                    double g = exp(-M->eta[s] * x * x);
                    sum += g * fc;
                    if (!useForces) continue;
                    double p1 = M->scalingFactor[s] * (dfc - 2.0 * M->eta[s] * x * fc) * g / n->d;
                    int row = M->row[s * NE + M->e1[s]];
                    for (int c = 0; c < 3; ++c)
                    {
                        gs[c] += p1 * n->dr[c];
                        n->dGdr[3 * row + c] -= p1 * n->dr[c];
                    }
                }
                R->G[R->sfOffset[i] + si] = scale_value(M, s, sum);
                continue;
            }
            /* angular: all pairs j < k of the neighbour list */
            int narrow = (M->type[s] == 3);
            double pnorm = pow(2.0, 1.0 - M->zeta[s]);
            double zl = M->zeta[s] * M->lambda[s];
            double fd = 2.0 * M->eta[s] / M->zeta[s] / M->lambda[s];
            int zint = (int)lround(M->zeta[s]);
            int useInt = fabs(M->zeta[s] - zint) <= 2.2250738585072014e-308;
            double fn = pnorm * M->scalingFactor[s];
            for (int64_t a = off[i]; a < off[i + 1]; ++a)
            {
                Nbr* nj = &nb[a];
                int ej = elem[nj->j];
                if (!((ej == M->e1[s] || ej == M->e2[s]) && nj->d < rcs)) continue;
                double fcij, dfcij;
                cutoff_fdf(M->cutoffType, M->cutoffAlpha, rcs, nj->d, &fcij, &dfcij);
                for (int64_t b = a + 1; b < off[i + 1]; ++b)
                {
                    Nbr* nk = &nb[b];
                    int ek = elem[nk->j];
                    if (!((M->e1[s] == ej && M->e2[s] == ek) || (M->e2[s] == ej && M->e1[s] == ek))) continue;
                    if (!(nk->d < rcs)) continue;
                    double d3[3] = {nk->dr[0] - nj->dr[0], nk->dr[1] - nj->dr[1], nk->dr[2] - nj->dr[2]};
                    double rjk2 = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
                    if (narrow && !(rjk2 < rcs * rcs)) continue;
                    double fcik, dfcik, fcjk = 1.0, dfcjk = 0.0, rjk = sqrt(rjk2);
                    cutoff_fdf(M->cutoffType, M->cutoffAlpha, rcs, nk->d, &fcik, &dfcik);
                    if (narrow) cutoff_fdf(M->cutoffType, M->cutoffAlpha, rcs, rjk, &fcjk, &dfcjk);
                    double rij = nj->d, rik = nk->d;
                    double rinv = 1.0 / rij / rik;
                    double cost = (nj->dr[0] * nk->dr[0] + nj->dr[1] * nk->dr[1] + nj->dr[2] * nk->dr[2]) * rinv;
                    double pfc = fcij * fcik * fcjk;
                    double xs = rij - M->rs[s], ys = rik - M->rs[s], zs = rjk - M->rs[s];
                    double arg = xs * xs + ys * ys + (narrow ? zs * zs : 0.0);
                    double vexp = exp(-M->eta[s] * arg);
                    double pl = 1.0 + M->lambda[s] * cost;
                    double fg = 0.0;
                    if (pl > 0.0)
                        fg = vexp * (useInt ? pow_by_squaring(pl, zint - 1) : pow(pl, M->zeta[s] - 1.0));
                    sum += fg * pl * pfc;
                    if (!useForces) continue;
                    double g = fg * fn;
                    double pfczl = pfc * zl;
                    double q = pl * fd;
                    double pr1 = fcik * fcjk * dfcij / rij;
                    double pr2 = fcij * fcjk * dfcik / rik;
                    double p1 = g * (pfczl * (rinv - cost / (rij * rij) - q * xs / rij) + pr1 * pl);
                    double p2 = g * (pfczl * (rinv - cost / (rik * rik) - q * ys / rik) + pr2 * pl);
                    double p3;
                    if (narrow)
                    {
                        double pr3 = fcij * fcik * dfcjk / rjk;
                        p3 = g * (pfczl * (rinv + q * zs / rjk) - pr3 * pl);
                    }
                    else p3 = g * pfczl * rinv;
                    int rj = M->row[s * NE + ej], rk = M->row[s * NE + ek];
                    for (int c = 0; c < 3; ++c)
                    {
                        gs[c] += p1 * nj->dr[c] + p2 * nk->dr[c];
                        nj->dGdr[3 * rj + c] -= p1 * nj->dr[c] + p3 * d3[c];
                        nk->dGdr[3 * rk + c] -= p2 * nk->dr[c] - p3 * d3[c];
                    }
                }
            }
            R->G[R->sfOffset[i] + si] = scale_value(M, s, sum * pnorm);
        }
        /* extrapolation check (Element.cpp:462-541) */
        for (int s = M->sfBegin[ec]; s < M->sfBegin[ec + 1]; ++s)
        {
            double v = unscale_value(M, s, R->G[R->sfOffset[i] + s - M->sfBegin[ec]]);
            double eps = 1000.0 * 2.220446049250313e-16;
            if (v + eps < M->Gmin[s] || v - eps > M->Gmax[s]) R->warnings++;
        }
    }
    /* atomic networks: forward and dE/dG */
    R->atomicEnergy = (double*)calloc(N > 0 ? N : 1, sizeof(double));
    double E = 0.0;
    for (int i = 0; i < N; ++i)
    {
        int ec = elem[i];
        int L = M->numLayers[ec];
        const int* nn = M->neurons + ec * 8;
        double* y[8];
        double* dy[8];
        for (int l = 0; l < L; ++l)
        {
            y[l] = (double*)calloc(nn[l], sizeof(double));
            dy[l] = (double*)calloc(nn[l], sizeof(double));
        }
        for (int k = 0; k < nn[0]; ++k) y[0][k] = R->G[R->sfOffset[i] + k];
        for (int l = 1; l < L; ++l)
        {
            const double* W = M->weights + M->wBegin[ec * 8 + l];
            const double* bb = M->weights + M->bBegin[ec * 8 + l];
            for (int k = 0; k < nn[l]; ++k)
            {
                double x = 0.0;
                for (int j = 0; j < nn[l - 1]; ++j) x += W[k * nn[l - 1] + j] * y[l - 1][j];
                x += bb[k];
                if (M->normalizeNeurons) x /= nn[l - 1];
                activation(M->activation[ec * 8 + l], x, &y[l][k], &dy[l][k]);
            }
        }
        R->atomicEnergy[i] = y[L - 1][0];
        E += y[L - 1][0];
        /* reverse accumulation of dE/dG */
        double* g = (double*)calloc(nn[L - 1], sizeof(double));
        g[0] = dy[L - 1][0] / (M->normalizeNeurons ? nn[L - 2] : 1);
        for (int l = L - 1; l >= 1; --l)
        {
            const double* W = M->weights + M->wBegin[ec * 8 + l];
            double* gp = (double*)calloc(nn[l - 1], sizeof(double));
            for (int j = 0; j < nn[l - 1]; ++j)
            {
                double t = 0.0;
                for (int k = 0; k < nn[l]; ++k) t += W[k * nn[l - 1] + j] * g[k];
                if (l > 1) t *= dy[l - 1][j] / (M->normalizeNeurons ? nn[l - 2] : 1);
                gp[j] = t;
            }
            free(g);
            g = gp;
        }
        for (int k = 0; k < nn[0]; ++k) R->dEdG[R->sfOffset[i] + k] = g[k];
        free(g);
        for (int l = 0; l < L; ++l)
        {
            free(y[l]);
            free(dy[l]);
        }
    }
    R->energyInternal = E;
    /* forces: self term plus, for every other atom j, all entries of j's
     * list that point at i (Mode::calculateForces semantics) */
    R->forces = (double*)calloc(3 * (N > 0 ? N : 1), sizeof(double));
    if (useForces)
    {
        for (int i = 0; i < N; ++i)
        {
            int ec = elem[i];
            double f[3] = {0, 0, 0};
            for (int s = 0; s < M->sfBegin[ec + 1] - M->sfBegin[ec]; ++s)
                for (int c = 0; c < 3; ++c) f[c] -= R->dEdG[R->sfOffset[i] + s] * dGself[3 * (R->sfOffset[i] + s) + c];
            int last = -1;
            for (int64_t e = off[i]; e < off[i + 1]; ++e)
            {
                int j = nb[e].j;
                if (j == i || j == last) continue;
                last = j;
                int ej = elem[j];
                for (int64_t q = off[j]; q < off[j + 1]; ++q)
                {
                    if (nb[q].j != i) continue;
                    int rows = M->numRows[ej * NE + ec];
                    const int* sfOfRow = M->rowSF + (ej * NE + ec) * M->maxRows;
                    for (int rr = 0; rr < rows; ++rr)
                        for (int c = 0; c < 3; ++c)
                            f[c] -= R->dEdG[R->sfOffset[j] + sfOfRow[rr]] * nb[q].dGdr[3 * rr + c];
                }
            }
            for (int c = 0; c < 3; ++c) R->forces[3 * i + c] = f[c];
        }
    }
    /* back to physical units */
    double Ephys = E;
    if (M->normalize)
    {
        Ephys = E / M->convEnergy + N * M->meanEnergy;
        double cf = M->convEnergy / M->convLength;
        for (int q = 0; q < 3 * N; ++q) R->forces[q] /= cf;
    }
    for (int e = 0; e < NE; ++e)
    {
        int cnt = 0;
        for (int i = 0; i < N; ++i) cnt += (elem[i] == e);
        Ephys += cnt * M->atomicEnergyOffset[e];
    }
    R->energy = Ephys;
    for (int64_t e = 0; e < M_; ++e) free(nb[e].dGdr);
    free(nb);
    free(dGself);
    return 0;
}
