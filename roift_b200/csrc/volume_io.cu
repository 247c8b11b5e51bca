// volume_io.cu -- host-side volume files of the reference CLI: gft::Scene32::Read / Write
// (gft/src/gft_scene32.cpp:334-420, 525-580, 600-660, 748-800) for .scn and NIfTI-1.
//
// .scn: "SCN\n", "X Y Z\n", "dx dy dz\n" (%f), the sample width (8, 16, 32) and one
//       separator byte, then little-endian samples; the writer picks 8 bits when the
//       maximum is below 256, 16 below 65536, else 32, and casts every value to that width.
// NIfTI-1: the 348-byte header (either byte order), data at max(vox_offset, 348) in a .nii
//       file or at vox_offset in the .img of a .hdr / .img pair; .nii.gz and .img.gz are read
//       and .nii.gz written through zlib.  Read conversions follow ReadNifti1: int32, uint16,
//       int16, uint8 and int8 are widened; float32 is scaled by 10000 / max (a float) and
//       rounded; complex, float64, RGB, 32/64-bit unsigned and wider types, and dim[0]
//       outside 3..4, are rejected.  The writer stores int32 samples (WriteNifti1) with
//       pixdim = spacing, qform / sform codes 0.
// Only the first volume of a 4D file is read (the reference copies all of them into a 3D
// buffer for int32 data).
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace {

bool ends_with(const std::string &s, const char *suffix) {
    const size_t n = std::strlen(suffix);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; i++) {
        char a = s[s.size() - n + i], b = suffix[i];
        if (a >= 'A' && a <= 'Z') a = (char)(a - 'A' + 'a');
        if (a != b) return false;
    }
    return true;
}

struct Nifti1Header {
    unsigned char raw[348];
    bool swap = false;
    template <typename T>
    T get(int off) const {
        T v;
        std::memcpy(&v, raw + off, sizeof(T));
        if (swap) {
            unsigned char *b = reinterpret_cast<unsigned char *>(&v);
            for (size_t i = 0; i < sizeof(T) / 2; i++) std::swap(b[i], b[sizeof(T) - 1 - i]);
        }
        return v;
    }
    template <typename T>
    void put(int off, T v) {
        std::memcpy(raw + off, &v, sizeof(T));
    }
};

// NIfTI-1 field offsets (nifti1.h)
constexpr int NH_SIZEOF = 0, NH_DIM = 40, NH_DATATYPE = 70, NH_BITPIX = 72, NH_PIXDIM = 76,
              NH_VOX_OFFSET = 108, NH_SCL_SLOPE = 112, NH_DESCRIP = 148, NH_QFORM = 252,
              NH_SFORM = 254, NH_MAGIC = 344;

int read_exact(gzFile f, void *dst, size_t bytes) {
    unsigned char *p = static_cast<unsigned char *>(dst);
    while (bytes > 0) {
        const unsigned chunk = bytes > (1u << 30) ? (1u << 30) : (unsigned)bytes;
        const int got = gzread(f, p, chunk);
        if (got <= 0) return -1;
        p += got;
        bytes -= (size_t)got;
    }
    return 0;
}

int read_scn(const std::string &path, int32_t *data, size_t cap, int dims[3], float sp[3]) {
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) return OIFT_E_BAD_ARG;
    char type[16] = {0};
    int X = 0, Y = 0, Z = 0, v = 0;
    float dx = 0, dy = 0, dz = 0;
    if (std::fscanf(fp, "%15s\n", type) != 1 || std::strcmp(type, "SCN") != 0 ||
        std::fscanf(fp, "%d %d %d\n", &X, &Y, &Z) != 3 ||
        std::fscanf(fp, "%f %f %f\n", &dx, &dy, &dz) != 3 || std::fscanf(fp, "%d", &v) != 1 ||
        X <= 0 || Y <= 0 || Z <= 0) {
        std::fclose(fp);
        return OIFT_E_BAD_ARG;
    }
    dims[0] = X;
    dims[1] = Y;
    dims[2] = Z;
    sp[0] = dx;
    sp[1] = dy;
    sp[2] = dz;
    const size_t n = (size_t)X * Y * Z;
    if (!data) {
        std::fclose(fp);
        return OIFT_OK;
    }
    if (cap < n) {
        std::fclose(fp);
        return OIFT_E_RANGE;
    }
    // the samples start one byte after the width (gft_scene32.cpp:372-374)
    const long pos = std::ftell(fp);
    std::fseek(fp, pos + 1, SEEK_SET);
    int rc = OIFT_OK;
    if (v == 8) {
        std::vector<unsigned char> b(n);
        if (std::fread(b.data(), 1, n, fp) != n) rc = OIFT_E_BAD_ARG;
        for (size_t i = 0; i < n && rc == OIFT_OK; i++) data[i] = (int32_t)b[i];
    } else if (v == 16) {
        std::vector<uint16_t> b(n);
        if (std::fread(b.data(), 2, n, fp) != n) rc = OIFT_E_BAD_ARG;
        for (size_t i = 0; i < n && rc == OIFT_OK; i++) data[i] = (int32_t)b[i];
    } else {
        if (std::fread(data, 4, n, fp) != n) rc = OIFT_E_BAD_ARG;
    }
    std::fclose(fp);
    return rc;
}

int write_scn(const std::string &path, const int32_t *data, const int dims[3], const float sp[3]) {
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) return OIFT_E_BAD_ARG;
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    std::fprintf(fp, "SCN\n%d %d %d\n%f %f %f\n", dims[0], dims[1], dims[2], sp[0], sp[1], sp[2]);
    int32_t imax = data[0];
    for (size_t i = 1; i < n; i++) imax = data[i] > imax ? data[i] : imax;
    bool ok;
    if (imax < 256) {
        std::fprintf(fp, "%d\n", 8);
        std::vector<unsigned char> b(n);
        for (size_t i = 0; i < n; i++) b[i] = (unsigned char)data[i];
        ok = std::fwrite(b.data(), 1, n, fp) == n;
    } else if (imax < 65536) {
        std::fprintf(fp, "%d\n", 16);
        std::vector<uint16_t> b(n);
        for (size_t i = 0; i < n; i++) b[i] = (uint16_t)data[i];
        ok = std::fwrite(b.data(), 2, n, fp) == n;
    } else {
        std::fprintf(fp, "%d\n", 32);
        ok = std::fwrite(data, 4, n, fp) == n;
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? OIFT_OK : OIFT_E_BAD_ARG;
}

// The data file of a NIfTI path: the path itself, or the .img of a .hdr (and the reverse).
std::string pair_name(const std::string &path, const char *from, const char *to) {
    const size_t n = std::strlen(from);
    std::string s = path.substr(0, path.size() - n);
    // keep the case of the extension's first letter, as a user would name the pair
    std::string ext = to;
    if (path[path.size() - n + 1] >= 'A' && path[path.size() - n + 1] <= 'Z')
        for (char &ch : ext) ch = (char)((ch >= 'a' && ch <= 'z') ? ch - 'a' + 'A' : ch);
    return s + ext;
}

int read_nifti(const std::string &path, int32_t *data, size_t cap, int dims[3], float sp[3]) {
    std::string hdr_path = path, img_path = path;
    if (ends_with(path, ".img")) hdr_path = pair_name(path, ".img", ".hdr");
    if (ends_with(path, ".img.gz")) hdr_path = pair_name(path, ".img.gz", ".hdr.gz");
    gzFile f = gzopen(hdr_path.c_str(), "rb");
    if (!f) return OIFT_E_BAD_ARG;
    Nifti1Header h;
    if (read_exact(f, h.raw, sizeof(h.raw)) != 0) {
        gzclose(f);
        return OIFT_E_BAD_ARG;
    }
    int32_t sz = h.get<int32_t>(NH_SIZEOF);
    if (sz != 348) {
        h.swap = true;
        sz = h.get<int32_t>(NH_SIZEOF);
    }
    if (sz != 348) {  // not NIfTI-1 / ANALYZE (NIfTI-2 has 540)
        gzclose(f);
        return OIFT_E_UNSUPPORTED;
    }
    const bool onefile = std::memcmp(h.raw + NH_MAGIC, "n+1", 4) == 0;
    int16_t dim[8];
    for (int i = 0; i < 8; i++) dim[i] = h.get<int16_t>(NH_DIM + 2 * i);
    const int dtype = h.get<int16_t>(NH_DATATYPE);
    if (dim[0] < 3 || dim[0] > 4) {
        gzclose(f);
        return OIFT_E_UNSUPPORTED;
    }
    int nb;
    switch (dtype) {
        case 2: case 256: nb = 1; break;       // uint8, int8
        case 4: case 512: nb = 2; break;       // int16, uint16
        case 8: case 16: nb = 4; break;        // int32, float32
        default: gzclose(f); return OIFT_E_UNSUPPORTED;
    }
    const int X = dim[1] < 1 ? 1 : dim[1], Y = dim[2] < 1 ? 1 : dim[2], Z = dim[3] < 1 ? 1 : dim[3];
    dims[0] = X;
    dims[1] = Y;
    dims[2] = Z;
    for (int k = 0; k < 3; k++) sp[k] = h.get<float>(NH_PIXDIM + 4 * (k + 1));
    const size_t n = (size_t)X * Y * Z;
    if (!data) {
        gzclose(f);
        return OIFT_OK;
    }
    if (cap < n) {
        gzclose(f);
        return OIFT_E_RANGE;
    }
    // data offset as nifti_image_read takes it (at least the header size in one file)
    long ioff = (long)(int)h.get<float>(NH_VOX_OFFSET);
    if (onefile) {
        if (ioff < 348) ioff = 348;
    } else {
        gzclose(f);
        if (ends_with(path, ".hdr")) img_path = pair_name(path, ".hdr", ".img");
        if (ends_with(path, ".hdr.gz")) img_path = pair_name(path, ".hdr.gz", ".img.gz");
        f = gzopen(img_path.c_str(), "rb");
        if (!f) return OIFT_E_BAD_ARG;
        if (ioff < 0) ioff = 0;
    }
    if (gzseek(f, ioff, SEEK_SET) != ioff) {
        gzclose(f);
        return OIFT_E_BAD_ARG;
    }
    std::vector<unsigned char> buf(n * (size_t)nb);
    const int rr = read_exact(f, buf.data(), buf.size());
    gzclose(f);
    if (rr != 0) return OIFT_E_BAD_ARG;
    auto sample = [&](size_t i, unsigned char *out) {
        std::memcpy(out, buf.data() + i * nb, nb);
        if (h.swap)
            for (int a = 0; a < nb / 2; a++) std::swap(out[a], out[nb - 1 - a]);
    };
    unsigned char s4[4];
    if (dtype == 16) {
        // ReadNifti1: float max = 0; factor = 10000.0 / max (a float); ROUND(v * factor)
        std::vector<float> v(n);
        float mx = 0.0f;
        for (size_t i = 0; i < n; i++) {
            sample(i, s4);
            std::memcpy(&v[i], s4, 4);
            if (mx < v[i]) mx = v[i];
        }
        if (!(mx > 0.0f)) return OIFT_E_RANGE;  // the reference divides by zero here
        const float factor = (float)(10000.0 / mx);
        for (size_t i = 0; i < n; i++) {
            const float x = v[i] * factor;
            data[i] = (x < 0) ? (int32_t)(x - 0.5) : (int32_t)(x + 0.5);
        }
        return OIFT_OK;
    }
    for (size_t i = 0; i < n; i++) {
        sample(i, s4);
        switch (dtype) {
            case 2: data[i] = (int32_t)s4[0]; break;
            case 256: data[i] = (int32_t)(signed char)s4[0]; break;
            case 4: { int16_t t; std::memcpy(&t, s4, 2); data[i] = t; break; }
            case 512: { uint16_t t; std::memcpy(&t, s4, 2); data[i] = t; break; }
            default: { int32_t t; std::memcpy(&t, s4, 4); data[i] = t; break; }
        }
    }
    return OIFT_OK;
}

int write_nifti(const std::string &path, const int32_t *data, const int dims[3], const float sp[3]) {
    const bool gz = ends_with(path, ".gz");
    const bool pair = ends_with(path, ".hdr") || ends_with(path, ".img") ||
                      ends_with(path, ".hdr.gz") || ends_with(path, ".img.gz");
    Nifti1Header h;
    std::memset(h.raw, 0, sizeof(h.raw));
    h.put<int32_t>(NH_SIZEOF, 348);
    const int16_t dim[8] = {3, (int16_t)dims[0], (int16_t)dims[1], (int16_t)dims[2], 1, 1, 1, 1};
    for (int i = 0; i < 8; i++) h.put<int16_t>(NH_DIM + 2 * i, dim[i]);
    h.put<int16_t>(NH_DATATYPE, 8);  // NIFTI_TYPE_INT32
    h.put<int16_t>(NH_BITPIX, 32);
    const float pixdim[8] = {1.0f, sp[0], sp[1], sp[2], 0, 0, 0, 0};
    for (int i = 0; i < 8; i++) h.put<float>(NH_PIXDIM + 4 * i, pixdim[i]);
    h.put<float>(NH_VOX_OFFSET, pair ? 0.0f : 352.0f);
    h.put<float>(NH_SCL_SLOPE, 0.0f);
    h.put<int16_t>(NH_QFORM, 0);
    h.put<int16_t>(NH_SFORM, 0);
    std::memcpy(h.raw + NH_MAGIC, pair ? "ni1\0" : "n+1\0", 4);
    (void)NH_DESCRIP;
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    const unsigned char ext[4] = {0, 0, 0, 0};
    auto put_file = [&](const std::string &name, bool header, bool body) -> bool {
        bool ok = true;
        if (gz) {
            gzFile f = gzopen(name.c_str(), "wb");
            if (!f) return false;
            if (header) ok = ok && gzwrite(f, h.raw, 348) == 348 && gzwrite(f, ext, 4) == 4;
            const unsigned char *p = reinterpret_cast<const unsigned char *>(data);
            size_t left = body ? n * 4 : 0;
            while (ok && left > 0) {
                const unsigned chunk = left > (1u << 30) ? (1u << 30) : (unsigned)left;
                ok = gzwrite(f, p, chunk) == (int)chunk;
                p += chunk;
                left -= chunk;
            }
            return (gzclose(f) == Z_OK) && ok;
        }
        FILE *f = std::fopen(name.c_str(), "wb");
        if (!f) return false;
        if (header) ok = ok && std::fwrite(h.raw, 1, 348, f) == 348 && std::fwrite(ext, 1, 4, f) == 4;
        if (body) ok = ok && std::fwrite(data, 4, n, f) == n;
        return (std::fclose(f) == 0) && ok;
    };
    if (!pair) return put_file(path, true, true) ? OIFT_OK : OIFT_E_BAD_ARG;
    std::string hdr = path, img = path;
    if (ends_with(path, ".img")) hdr = pair_name(path, ".img", ".hdr");
    if (ends_with(path, ".img.gz")) hdr = pair_name(path, ".img.gz", ".hdr.gz");
    if (ends_with(path, ".hdr")) img = pair_name(path, ".hdr", ".img");
    if (ends_with(path, ".hdr.gz")) img = pair_name(path, ".hdr.gz", ".img.gz");
    return (put_file(hdr, true, false) && put_file(img, false, true)) ? OIFT_OK : OIFT_E_BAD_ARG;
}

bool is_nifti(const std::string &p) {
    return ends_with(p, ".nii") || ends_with(p, ".nii.gz") || ends_with(p, ".hdr") ||
           ends_with(p, ".img") || ends_with(p, ".hdr.gz") || ends_with(p, ".img.gz");
}

}  // namespace

extern "C" {

OIFT_API int oift_b200_read_volume(const char *path, int32_t *data, size_t cap_voxels,
                                   int dims[3], float spacing[3]) {
    if (!path || !dims || !spacing) return OIFT_E_BAD_ARG;
    const std::string p(path);
    if (ends_with(p, ".scn")) return read_scn(p, data, cap_voxels, dims, spacing);
    if (is_nifti(p)) return read_nifti(p, data, cap_voxels, dims, spacing);
    return OIFT_E_UNSUPPORTED;
}

OIFT_API int oift_b200_write_volume(const char *path, const int32_t *data, const int dims[3],
                                    const float spacing[3]) {
    if (!path || !data || !dims || !spacing) return OIFT_E_BAD_ARG;
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return OIFT_E_BAD_ARG;
    const std::string p(path);
    if (ends_with(p, ".scn")) return write_scn(p, data, dims, spacing);
    if (is_nifti(p)) {
        if (dims[0] > 32767 || dims[1] > 32767 || dims[2] > 32767) return OIFT_E_RANGE;
        return write_nifti(p, data, dims, spacing);
    }
    return OIFT_E_UNSUPPORTED;
}

}  // extern "C"
