// Host-side file formats of the registration path, written and read the way
// Plastimatch does so files move between the two unchanged:
//   B-spline coefficients  Bspline_xform::save / bspline_xform_load
//                          (src/base/bspline_xform.cxx:101-279): a text
//                          header of key = value lines, then the
//                          coefficients one per line, x of every knot,
//                          then y, then z ("ITK-like planar")
//   MetaImage (.mha)       write_mha / read_mha (src/base/mha_io.cxx:
//                          25-241): the reference's header lines, then raw
//                          little-endian samples; float images and
//                          interleaved 3-channel vector fields are written,
//                          float, short and unsigned char are read (and
//                          converted to float)
// Host memory only; these functions make no CUDA call.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/plastimatch_b200.h"

namespace b200 {
int static_fail (int code, const char* msg);   // runtime.cu
}

using b200::static_fail;

namespace {

struct File {
    FILE* fp;
    explicit File (FILE* f) : fp (f) {}
    ~File () { if (fp) fclose (fp); }
};

// Bspline_header::set (src/base/bspline_header.cxx:28-62)
int64_t
grid_coeffs (const b200bsp_grid* g)
{
    int64_t n = 3;
    for (int d = 0; d < 3; d++) {
        if (g->vox_per_rgn[d] < 1 || g->roi_dim[d] < 1) return -1;
        n *= 1 + (g->roi_dim[d] - 1) / g->vox_per_rgn[d] + 3;
    }
    return n;
}

bool
getline_c (FILE* fp, std::string& s)
{
    s.clear ();
    int c;
    bool any = false;
    while ((c = fgetc (fp)) != EOF) {
        any = true;
        if (c == '\n') break;
        s.push_back ((char) c);
    }
    return any;
}

void
rtrim (std::string& s)
{
    while (!s.empty () && (s.back () == ' ' || s.back () == '\t'
        || s.back () == '\r' || s.back () == '\n')) {
        s.pop_back ();
    }
}

bool
starts_with (const std::string& s, const char* p)
{
    return s.compare (0, strlen (p), p) == 0;
}

} // namespace

extern "C" int
b200bsp_xform_save (const char* path, const b200bsp_volume* fixed,
    const b200bsp_grid* grid, const float* coeff)
{
    if (!path || !fixed || !grid || !coeff) {
        return static_fail (B200BSP_E_BADARG, "null argument");
    }
    const int64_t n = grid_coeffs (grid);
    if (n < 0) return static_fail (B200BSP_E_BADARG, "bad grid");
    File f (fopen (path, "wb"));
    if (!f.fp) return static_fail (B200BSP_E_IO, "cannot open file for writing");
    FILE* fp = f.fp;
    fprintf (fp, "MGH_GPUIT_BSP <experimental>\n");
    fprintf (fp, "img_origin = %f %f %f\n", fixed->origin[0], fixed->origin[1],
        fixed->origin[2]);
    fprintf (fp, "img_spacing = %f %f %f\n", fixed->spacing[0],
        fixed->spacing[1], fixed->spacing[2]);
    fprintf (fp, "img_dim = %u %u %u\n", (unsigned) fixed->dim[0],
        (unsigned) fixed->dim[1], (unsigned) fixed->dim[2]);
    fprintf (fp, "roi_offset = %d %d %d\n", (int) grid->roi_offset[0],
        (int) grid->roi_offset[1], (int) grid->roi_offset[2]);
    fprintf (fp, "roi_dim = %d %d %d\n", (int) grid->roi_dim[0],
        (int) grid->roi_dim[1], (int) grid->roi_dim[2]);
    fprintf (fp, "vox_per_rgn = %d %d %d\n", (int) grid->vox_per_rgn[0],
        (int) grid->vox_per_rgn[1], (int) grid->vox_per_rgn[2]);
    const float* dc = fixed->dcos;
    fprintf (fp, "direction_cosines = %f %f %f %f %f %f %f %f %f\n", dc[0],
        dc[1], dc[2], dc[3], dc[4], dc[5], dc[6], dc[7], dc[8]);
    for (int c = 0; c < 3; c++) {
        for (int64_t k = 0; k < n / 3; k++) {
            fprintf (fp, "%.20f\n", coeff[3 * k + c]);
        }
    }
    if (ferror (fp)) return static_fail (B200BSP_E_IO, "write failed");
    return B200BSP_OK;
}

extern "C" int
b200bsp_xform_load (const char* path, b200bsp_volume* fixed,
    b200bsp_grid* grid, float* coeff, int64_t coeff_cap, int64_t* num_coeff)
{
    if (!path || !fixed || !grid) return static_fail (B200BSP_E_BADARG, "null argument");
    File f (fopen (path, "rb"));
    if (!f.fp) return static_fail (B200BSP_E_IO, "cannot open file");
    std::string line;
    if (!getline_c (f.fp, line) || !starts_with (line, "MGH_GPUIT_BSP")) {
        return static_fail (B200BSP_E_IO, "not a B-spline coefficient file");
    }
    b200bsp_volume v;
    b200bsp_grid g;
    memset (&v, 0, sizeof v);
    memset (&g, 0, sizeof g);
    for (int d = 0; d < 3; d++) v.spacing[d] = 1.f;
    v.dcos[0] = v.dcos[4] = v.dcos[8] = 1.f;
    // header lines until the first line without '=' (the first coefficient)
    while (true) {
        if (!getline_c (f.fp, line)) {
            return static_fail (B200BSP_E_IO, "truncated header");
        }
        if (line.find ('=') == std::string::npos) break;
        float a[9];
        unsigned u[3];
        const char* s = line.c_str ();
        if (sscanf (s, "img_origin = %f %f %f", &a[0], &a[1], &a[2]) == 3) {
            for (int d = 0; d < 3; d++) v.origin[d] = a[d];
        } else if (sscanf (s, "img_spacing = %f %f %f", &a[0], &a[1], &a[2]) == 3) {
            for (int d = 0; d < 3; d++) v.spacing[d] = a[d];
        } else if (sscanf (s, "img_dim = %u %u %u", &u[0], &u[1], &u[2]) == 3) {
            for (int d = 0; d < 3; d++) v.dim[d] = u[d];
        } else if (sscanf (s, "roi_offset = %u %u %u", &u[0], &u[1], &u[2]) == 3) {
            for (int d = 0; d < 3; d++) g.roi_offset[d] = u[d];
        } else if (sscanf (s, "roi_dim = %u %u %u", &u[0], &u[1], &u[2]) == 3) {
            for (int d = 0; d < 3; d++) g.roi_dim[d] = u[d];
        } else if (sscanf (s, "vox_per_rgn = %u %u %u", &u[0], &u[1], &u[2]) == 3) {
            for (int d = 0; d < 3; d++) g.vox_per_rgn[d] = u[d];
        } else if (sscanf (s, "direction_cosines = %f %f %f %f %f %f %f %f %f",
                       &a[0], &a[1], &a[2], &a[3], &a[4], &a[5], &a[6], &a[7],
                       &a[8]) == 9) {
            for (int i = 0; i < 9; i++) v.dcos[i] = a[i];
        } else {
            return static_fail (B200BSP_E_IO, "unknown header line");
        }
    }
    const int64_t n = grid_coeffs (&g);
    if (n < 3) return static_fail (B200BSP_E_IO, "header gives no coefficients");
    *fixed = v;
    *grid = g;
    if (num_coeff) *num_coeff = n;
    if (!coeff) return B200BSP_OK;
    if (coeff_cap < n) {
        return static_fail (B200BSP_E_BADARG, "coefficient buffer too small");
    }
    // planar order: all x, then all y, then all z; the first value is on
    // the line already read
    for (int c = 0; c < 3; c++) {
        for (int64_t k = 0; k < n / 3; k++) {
            if ((c != 0 || k != 0) && !getline_c (f.fp, line)) {
                return static_fail (B200BSP_E_IO, "too few coefficients");
            }
            if (sscanf (line.c_str (), "%f", &coeff[3 * k + c]) != 1) {
                return static_fail (B200BSP_E_IO, "bad coefficient line");
            }
        }
    }
    return B200BSP_OK;
}

extern "C" int
b200bsp_mha_write (const char* path, const b200bsp_volume* g, int channels,
    const float* data)
{
    if (!path || !g || !data) return static_fail (B200BSP_E_BADARG, "null argument");
    if (channels != 1 && channels != 3) {
        return static_fail (B200BSP_E_BADARG, "channels must be 1 or 3");
    }
    File f (fopen (path, "wb"));
    if (!f.fp) return static_fail (B200BSP_E_IO, "cannot open file for writing");
    const float* dc = g->dcos;
    fprintf (f.fp,
        "ObjectType = Image\n"
        "NDims = 3\n"
        "BinaryData = True\n"
        "BinaryDataByteOrderMSB = False\n"
        "TransformMatrix = %g %g %g %g %g %g %g %g %g\n"
        "Offset = %g %g %g\n"
        "CenterOfRotation = 0 0 0\n"
        "ElementSpacing = %g %g %g\n"
        "DimSize = %d %d %d\n"
        "AnatomicalOrientation = RAI\n"
        "%s"
        "ElementType = MET_FLOAT\n"
        "ElementDataFile = LOCAL\n",
        dc[0], dc[3], dc[6], dc[1], dc[4], dc[7], dc[2], dc[5], dc[8],
        g->origin[0], g->origin[1], g->origin[2],
        g->spacing[0], g->spacing[1], g->spacing[2],
        (int) g->dim[0], (int) g->dim[1], (int) g->dim[2],
        channels == 3 ? "ElementNumberOfChannels = 3\n" : "");
    const size_t n = (size_t) g->dim[0] * g->dim[1] * g->dim[2] * channels;
    if (fwrite (data, sizeof (float), n, f.fp) != n) {
        return static_fail (B200BSP_E_IO, "write failed");
    }
    return B200BSP_OK;
}

extern "C" int
b200bsp_mha_read (const char* path, b200bsp_volume* g, int* channels,
    float* data, int64_t cap)
{
    if (!path || !g || !channels) return static_fail (B200BSP_E_BADARG, "null argument");
    File f (fopen (path, "rb"));
    if (!f.fp) return static_fail (B200BSP_E_IO, "cannot open file");
    b200bsp_volume v;
    memset (&v, 0, sizeof v);
    v.dcos[0] = v.dcos[4] = v.dcos[8] = 1.f;
    // element kinds as read_mha tracks them
    enum { UNDEF, FLOAT, VF, SHORT, UCHAR } kind = UNDEF;
    bool msb = false, have_data = false;
    std::string line;
    while (getline_c (f.fp, line)) {
        rtrim (line);
        if (line == "ElementDataFile = LOCAL") {
            have_data = true;
            break;
        }
        const char* s = line.c_str ();
        unsigned u[3];
        float a[9];
        int tmp;
        if (sscanf (s, "DimSize = %u %u %u", &u[0], &u[1], &u[2]) == 3) {
            for (int d = 0; d < 3; d++) v.dim[d] = u[d];
        } else if (sscanf (s, "Offset = %g %g %g", &a[0], &a[1], &a[2]) == 3) {
            for (int d = 0; d < 3; d++) v.origin[d] = a[d];
        } else if (sscanf (s, "ElementSpacing = %g %g %g", &a[0], &a[1], &a[2]) == 3) {
            for (int d = 0; d < 3; d++) v.spacing[d] = a[d];
        } else if (sscanf (s, "TransformMatrix = %g %g %g %g %g %g %g %g %g",
                       &a[0], &a[3], &a[6], &a[1], &a[4], &a[7], &a[2], &a[5],
                       &a[8]) == 9) {
            for (int i = 0; i < 9; i++) v.dcos[i] = a[i];
        } else if (sscanf (s, "ElementNumberOfChannels = %d", &tmp) == 1) {
            if (kind == UNDEF || kind == FLOAT) kind = VF;
        } else if (line == "ElementType = MET_FLOAT") {
            if (kind == UNDEF) kind = FLOAT;
        } else if (line == "ElementType = MET_SHORT") {
            kind = SHORT;
        } else if (line == "ElementType = MET_UCHAR") {
            kind = UCHAR;
        } else if (line == "BinaryDataByteOrderMSB = True") {
            msb = true;
        }
    }
    if (!have_data) return static_fail (B200BSP_E_IO, "no local data section");
    if (kind == UNDEF) return static_fail (B200BSP_E_IO, "unsupported element type");
    const int ch = kind == VF ? 3 : 1;
    *g = v;
    *channels = ch;
    if (!data) return B200BSP_OK;
    const size_t npix = (size_t) v.dim[0] * v.dim[1] * v.dim[2];
    if (cap < (int64_t) (npix * ch)) {
        return static_fail (B200BSP_E_BADARG, "data buffer too small");
    }
    const size_t esize = kind == SHORT ? 2 : kind == UCHAR ? 1 : 4;
    const size_t count = npix * ch;
    std::vector<unsigned char> raw (count * esize);
    if (fread (raw.data (), esize, count, f.fp) != count) {
        return static_fail (B200BSP_E_IO, "short read");
    }
    if (msb && esize > 1) {
        for (size_t i = 0; i < count; i++) {
            unsigned char* p = &raw[i * esize];
            for (size_t b = 0; b < esize / 2; b++) {
                std::swap (p[b], p[esize - 1 - b]);
            }
        }
    }
    for (size_t i = 0; i < count; i++) {
        if (esize == 4) {
            memcpy (&data[i], &raw[4 * i], 4);
        } else if (esize == 2) {
            int16_t x;
            memcpy (&x, &raw[2 * i], 2);
            data[i] = (float) x;
        } else {
            data[i] = (float) raw[i];
        }
    }
    return B200BSP_OK;
}
