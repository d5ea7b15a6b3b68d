/* Forced-include prelude for compiling Plastimatch's B-spline cost-function
 * sources as a CPU test oracle without ITK.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this.
 *
 * The reference sources are compiled where they lie (read-only).  A few of
 * their headers pull in ITK (itkMatrix.h, itkImage.h ...), which is not
 * installed.  Because quoted includes resolve next to the including file
 * first, those headers cannot be replaced by an -I directory.  Instead this
 * prelude is force-included (-include) into every translation unit: it
 * defines the include guards of the ITK-facing headers and provides the few
 * types the cost-function path actually touches:
 *
 *   itk_direction_type.h  -> DirectionType (3x3 double matrix, row access)
 *   itk_image*.h          -> nothing (unused on the path)
 *   plm_image.h           -> Plm_image with a shared-pointer typedef
 *   plm_image_header.h    -> Plm_image_header holding dim/origin/spacing/dcos
 *
 * None of these stand-ins contain reference code; they only satisfy the
 * declarations used by volume_header.cxx / bspline_header.cxx /
 * bspline_xform.cxx. */
#ifndef ORACLE_REF_PRELUDE_H
#define ORACLE_REF_PRELUDE_H

#ifdef __cplusplus
#include <memory>
#include <string.h>
#include <stdint.h>

#define _itk_direction_type_h_
#define _itk_image_h_
#define _itk_image_type_h_
#define _itk_image_region_h_
#define _itk_image_origin_h_
#define _plm_image_h_
#define _plm_image_header_h_

namespace itk {
template<class T, unsigned int NRows, unsigned int NColumns>
class Matrix {
public:
    T m[NRows][NColumns];
    T* operator[] (unsigned int r) { return m[r]; }
    const T* operator[] (unsigned int r) const { return m[r]; }
};
}
typedef itk::Matrix<double, 3, 3> DirectionType;

class Plm_image {
public:
    typedef std::shared_ptr<Plm_image> Pointer;
};

class Volume;
class Volume_header;
class Bspline_xform;

/* Geometry-only image header: the cost-function path reads it through
 * get_dim / get_origin / get_spacing / get_direction_cosines. */
class Plm_image_header {
public:
    int64_t dim_[3];
    float origin_[3];
    float spacing_[3];
    float dc_[9];
    Plm_image_header () {
        for (int d = 0; d < 3; d++) {
            dim_[d] = 0; origin_[d] = 0.f; spacing_[d] = 1.f;
        }
        for (int i = 0; i < 9; i++) dc_[i] = (i % 4 == 0) ? 1.f : 0.f;
    }
    Plm_image_header (const int64_t d[3], const float o[3],
        const float s[3], const float* dc) {
        set_dim (d); set_origin (o); set_spacing (s);
        set_direction_cosines (dc);
    }
    explicit Plm_image_header (const Plm_image::Pointer&)
        : Plm_image_header () {}
    /* Row-accessible direction matrix, as ITK's GetDirection() returns. */
    DirectionType GetDirection () const {
        DirectionType m;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) m[r][c] = dc_[3*r+c];
        return m;
    }
    void get_origin (float o[3]) const { memcpy (o, origin_, sizeof origin_); }
    void get_spacing (float s[3]) const { memcpy (s, spacing_, sizeof spacing_); }
    void get_dim (int64_t d[3]) const { memcpy (d, dim_, sizeof dim_); }
    void get_direction_cosines (float dc[9]) const { memcpy (dc, dc_, sizeof dc_); }
    void set_dim (const int64_t d[3]) { memcpy (dim_, d, sizeof dim_); }
    void set_origin (const float o[3]) { memcpy (origin_, o, sizeof origin_); }
    void set_spacing (const float s[3]) { memcpy (spacing_, s, sizeof spacing_); }
    void set_direction_cosines (const float dc[9]) { memcpy (dc_, dc, sizeof dc_); }
};

#endif /* __cplusplus */
#endif
