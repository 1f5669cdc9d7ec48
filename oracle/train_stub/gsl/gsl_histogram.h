// Stand-in for the GSL histogram the reference's Dataset uses for its
// symmetry-function histograms (not on the training path), written for this
// project and used ONLY to compile the reference's nnp-train into the test
// oracle: uniform bins, increment, fprintf of "lower upper count" lines.
#ifndef N2P2B200_GSL_HISTOGRAM_STUB_H
#define N2P2B200_GSL_HISTOGRAM_STUB_H

#include <cstddef>
#include <cstdio>

struct gsl_histogram
{
    std::size_t n;
    double*     range;
    double*     bin;
};

inline gsl_histogram* gsl_histogram_alloc(std::size_t n)
{
    gsl_histogram* h = new gsl_histogram();
    h->n = n;
    h->range = new double[n + 1]();
    h->bin = new double[n]();
    return h;
}

inline int gsl_histogram_set_ranges_uniform(gsl_histogram* h, double xmin, double xmax)
{
    for (std::size_t i = 0; i <= h->n; ++i) h->range[i] = xmin + (xmax - xmin) * (double)i / (double)h->n;
    for (std::size_t i = 0; i < h->n; ++i) h->bin[i] = 0.0;
    return 0;
}

inline int gsl_histogram_increment(gsl_histogram* h, double x)
{
    if (!(x >= h->range[0] && x < h->range[h->n])) return 1;
    std::size_t i = 0;
    while (i + 1 < h->n && x >= h->range[i + 1]) ++i;
    h->bin[i] += 1.0;
    return 0;
}

inline int gsl_histogram_fprintf(FILE* f, const gsl_histogram* h, const char* rf, const char* bf)
{
    for (std::size_t i = 0; i < h->n; ++i)
    {
        std::fprintf(f, rf, h->range[i]);
        std::fprintf(f, " ");
        std::fprintf(f, rf, h->range[i + 1]);
        std::fprintf(f, " ");
        std::fprintf(f, bf, h->bin[i]);
        std::fprintf(f, "\n");
    }
    return 0;
}

inline void gsl_histogram_free(gsl_histogram* h)
{
    delete[] h->range;
    delete[] h->bin;
    delete h;
}

#endif
