/*
 * field_layout.hpp -- drop-in replacement for bfps/cpp/field_layout.hpp
 * (bfps_b200: the device engine behind include/bfps_b200.h).
 *
 * Same names and members as the reference (field_layout.hpp:30-106): the
 * component enum, ncomp / ndim, and the size / subsize / start description
 * of a field's local slab.  One process holds the whole grid here (no MPI
 * slabs), so subsizes == sizes and starts == 0.  MPI, HDF5 and FFTW types
 * that appear in the reference signatures are taken from their own headers
 * when those were included first (a bfps build), else given minimal
 * stand-ins so that the classes also build without them.
 */
#ifndef BFPS_B200_FIELD_LAYOUT_HPP
#define BFPS_B200_FIELD_LAYOUT_HPP

#include <cstdint>
#include <cstddef>

#ifndef MPI_VERSION
typedef int MPI_Comm;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
#endif
#ifndef H5_VERS_MAJOR
typedef int64_t hid_t;
typedef unsigned long long hsize_t;
#endif
#ifndef FFTW_MEASURE
#define FFTW_MEASURE (0U)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#endif
#ifndef DEFAULT_FFTW_FLAG
#define DEFAULT_FFTW_FLAG FFTW_ESTIMATE
#endif

enum field_backend { FFTW };
enum field_components { ONE, THREE, THREExTHREE };

constexpr unsigned int ncomp(field_components fc) {
    return ((fc == THREE) ? 3 : ((fc == THREExTHREE) ? 9 : 1));
}
constexpr unsigned int ndim(field_components fc) {
    return ((fc == THREE) ? 4 : ((fc == THREExTHREE) ? 5 : 3));
}

template <field_components fc>
class field_layout {
  public:
    hsize_t sizes[ndim(fc)];
    hsize_t subsizes[ndim(fc)];
    hsize_t starts[ndim(fc)];
    hsize_t local_size, full_size;
    int myrank = 0, nprocs = 1;
    MPI_Comm comm;

    field_layout(const hsize_t* SIZES, const hsize_t* SUBSIZES, const hsize_t* STARTS,
                 const MPI_Comm COMM_TO_USE)
        : comm(COMM_TO_USE) {
        local_size = 1;
        full_size = 1;
        for (int i = 0; i < 3; ++i) {
            sizes[i] = SIZES[i];
            subsizes[i] = SUBSIZES[i];
            starts[i] = STARTS[i];
            local_size *= subsizes[i];
            full_size *= sizes[i];
        }
        if (fc == THREE) {
            sizes[3] = subsizes[3] = 3;
            starts[3] = 0;
            local_size *= 3;
            full_size *= 3;
        } else if (fc == THREExTHREE) {
            sizes[3] = subsizes[3] = sizes[4] = subsizes[4] = 3;
            starts[3] = starts[4] = 0;
            local_size *= 9;
            full_size *= 9;
        }
    }
};

#endif
