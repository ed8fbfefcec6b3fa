// persist.cu -- reading and writing saved matrices in the reference's binary persistence format, so
// that matrices a Pascal program saved (and the reference's own test fixtures) feed the GPU path.
//
// Format (TBinaryReaderWriter, BinaryReaderWriter.pas; object model BaseMathPersistence.pas): the
// 5-byte header "RMCLS", a uint32 version (1), then sections, each a packed record {int32 total
// length, uint8 section type, uint16 name length} followed by the UTF-8 name and the payload, up to
// an end-of-stream section.  A TDoubleMatrix (class identifier "MTX", DblMatrix.pas:3403) writes an
// object-description section ("obj" = "MTX"), then the properties of TBaseMatrix.DefineProps
// (Matrix.pas:873-887): string Name, integers Width and Height, the double array "data" (the full
// matrix row by row, DblMatrix.pas:3354-3367) and integers SubWidth, SubHeight, OffsetX, OffsetY
// (the sub-matrix view).  Property names compare case-insensitively (CompareText), unknown ones are
// skipped, as the reference's OnLoad* handlers do.  The writer emits the sections in the order of the
// reference's saved fixtures, so that it reproduces them byte for byte.
#include <cstdio>
#include <cstring>
#include <string>
#include <strings.h>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

enum SectType : uint8_t {  // TBinarySectionType (BinaryReaderWriter.pas), one byte ({$MINENUMSIZE 1})
    kBsBinary = 0, kBsString, kBsDouble, kBsDoubleArr, kBsIntArr, kBsInteger, kBsBeginList, kBsListIntArr,
    kBsListDoubleArr, kBsEndList, kBsObjectDescription, kBsObjectBegin, kBsObjectEnd, kBsEndaStream, kBsComplex,
    kBsComplexArr
};
constexpr int kSectHeader = 7;  // packed {int32, uint8, uint16}

struct Parsed {
    int64_t width = -1, height = -1, sub_w = -1, sub_h = -1, off_x = 0, off_y = 0;
    std::vector<double> data;
};

int32_t parse_matrix(const std::vector<unsigned char>& raw, Parsed* out) {
    if (raw.size() < 9 || std::memcmp(raw.data(), "RMCLS", 5) != 0) return B2M_ERR_FORMAT;
    size_t pos = 9;
    bool is_mtx = false, ended = false;
    while (pos + kSectHeader <= raw.size()) {
        int32_t len;
        uint16_t nlen;
        std::memcpy(&len, &raw[pos], 4);
        const uint8_t typ = raw[pos + 4];
        std::memcpy(&nlen, &raw[pos + 5], 2);
        if (len < kSectHeader + nlen || pos + (size_t)len > raw.size()) return B2M_ERR_FORMAT;
        const std::string name(reinterpret_cast<const char*>(&raw[pos + kSectHeader]), nlen);
        const unsigned char* payload = &raw[pos + kSectHeader + nlen];
        const size_t plen = (size_t)len - kSectHeader - nlen;
        switch (typ) {
            case kBsObjectDescription: {
                // TDoubleMatrix ("MTX"), TThreadedMatrix ("TMTX", ThreadedMatrix.pas:115-118) and the
                // TB2MMatrix class of the Pascal binding ("B2MMTX") save the same properties
                const std::string cls(reinterpret_cast<const char*>(payload), plen);
                is_mtx = cls == "MTX" || cls == "TMTX" || cls == "B2MMTX";
                if (!is_mtx) return B2M_ERR_FORMAT;  // another persisted class
                break;
            }
            case kBsInteger: {
                if (plen != 4) return B2M_ERR_FORMAT;
                int32_t v;
                std::memcpy(&v, payload, 4);
                const char* nm = name.c_str();
                if (!strcasecmp(nm, "Width")) out->width = v;
                else if (!strcasecmp(nm, "Height")) out->height = v;
                else if (!strcasecmp(nm, "SubWidth")) out->sub_w = v;
                else if (!strcasecmp(nm, "SubHeight")) out->sub_h = v;
                else if (!strcasecmp(nm, "OffsetX")) out->off_x = v;
                else if (!strcasecmp(nm, "OffsetY")) out->off_y = v;
                break;
            }
            case kBsDoubleArr:
                if (plen % 8) return B2M_ERR_FORMAT;
                if (!strcasecmp(name.c_str(), "data")) {
                    out->data.resize(plen / 8);
                    if (plen) std::memcpy(out->data.data(), payload, plen);
                }
                break;
            case kBsObjectBegin:
            case kBsBeginList:
                return B2M_ERR_FORMAT;  // nested objects and lists are not part of a saved matrix
            case kBsEndaStream:
                ended = true;
                break;
            default:
                break;  // other properties (Name, ...) carry nothing the matrix needs
        }
        pos += (size_t)len;
        if (ended) break;
    }
    if (!ended || !is_mtx || out->width < 0 || out->height < 0) return B2M_ERR_FORMAT;
    if ((int64_t)out->data.size() != out->width * out->height) return B2M_ERR_FORMAT;  // OnLoadDoubleArr check
    if (out->sub_w < 0) out->sub_w = out->width;
    if (out->sub_h < 0) out->sub_h = out->height;
    return B2M_OK;
}

int32_t load_file(const char* path, Parsed* p) {
    if (!path) return B2M_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return B2M_ERR_ARG;
    std::vector<unsigned char> raw;
    unsigned char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) raw.insert(raw.end(), buf, buf + got);
    std::fclose(f);
    return parse_matrix(raw, p);
}

void put_section(std::vector<unsigned char>& o, uint8_t typ, const char* name, const void* payload, size_t plen) {
    const uint16_t nlen = (uint16_t)std::strlen(name);
    const int32_t len = (int32_t)(kSectHeader + nlen + plen);
    const unsigned char* l = reinterpret_cast<const unsigned char*>(&len);
    o.insert(o.end(), l, l + 4);
    o.push_back(typ);
    const unsigned char* n = reinterpret_cast<const unsigned char*>(&nlen);
    o.insert(o.end(), n, n + 2);
    o.insert(o.end(), name, name + nlen);
    const unsigned char* p = static_cast<const unsigned char*>(payload);
    if (plen) o.insert(o.end(), p, p + plen);
}

void put_int(std::vector<unsigned char>& o, const char* name, int64_t v) {
    const int32_t x = (int32_t)v;
    put_section(o, kBsInteger, name, &x, 4);
}

void fill_info(const Parsed& p, b2m_matrix_info* info) {
    info->width = p.width;
    info->height = p.height;
    info->sub_width = p.sub_w;
    info->sub_height = p.sub_h;
    info->offset_x = p.off_x;
    info->offset_y = p.off_y;
}

}  // namespace
}  // namespace b2m

using namespace b2m;

extern "C" int32_t b2m_ReadMatrixFile(const char* path, b2m_matrix_info* info, double* dst, int64_t LineWidth) {
    if (!info) return B2M_ERR_ARG;
    Parsed p;
    B2M_TRY(load_file(path, &p));
    fill_info(p, info);
    if (!dst) return B2M_OK;  // size query
    if (LineWidth < p.width * 8 || (LineWidth % 8)) return B2M_ERR_DIM;
    for (int64_t r = 0; r < p.height; ++r)
        std::memcpy(reinterpret_cast<char*>(dst) + r * LineWidth, p.data.data() + r * p.width, (size_t)p.width * 8);
    return B2M_OK;
}

extern "C" int32_t b2m_dev_ReadMatrixFile(b2m_ctx* h, const char* path, b2m_matrix_info* info, double* dst,
                                          int64_t LineWidth) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || !info) return B2M_ERR_ARG;
    Parsed p;
    const int32_t r = load_file(path, &p);
    if (r != B2M_OK) return fail(ctx, r, "b2m_dev_ReadMatrixFile: %s is not a readable saved matrix", path);
    fill_info(p, info);
    if (!dst) return B2M_OK;
    if (LineWidth < p.width * 8 || (LineWidth % 8)) return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (p.width == 0 || p.height == 0) return B2M_OK;
    CallLock lk(ctx);
    cudaSetDevice(ctx->device);
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, LineWidth, p.data.data(), p.width * 8, p.width * 8, p.height,
                                  cudaMemcpyHostToDevice, ctx->stream));
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));  // the host copy goes out of scope
    return B2M_OK;
}

extern "C" int32_t b2m_WriteMatrixFile(const char* path, const double* src, int64_t LineWidth, int64_t width,
                                       int64_t height) {
    if (!path || (!src && width * height > 0)) return B2M_ERR_ARG;
    if (width < 0 || height < 0 || width > 0x7fffffff || height > 0x7fffffff) return B2M_ERR_DIM;
    if (height > 0 && (LineWidth < width * 8 || (LineWidth % 8))) return B2M_ERR_DIM;
    if (width * height * 8 + 64 > 0x7fffffffll) return B2M_ERR_UNSUPPORTED;  // one int32-sized section
    std::vector<unsigned char> o;
    const char head[5] = {'R', 'M', 'C', 'L', 'S'};
    o.insert(o.end(), head, head + 5);
    const uint32_t version = 1;
    const unsigned char* v = reinterpret_cast<const unsigned char*>(&version);
    o.insert(o.end(), v, v + 4);
    put_section(o, kBsObjectDescription, "obj", "MTX", 3);
    put_section(o, kBsString, "Name", nullptr, 0);
    put_int(o, "Width", width);
    put_int(o, "Height", height);
    std::vector<double> data((size_t)(width * height));
    for (int64_t r = 0; r < height; ++r)
        std::memcpy(data.data() + r * width, reinterpret_cast<const char*>(src) + r * LineWidth, (size_t)width * 8);
    put_section(o, kBsDoubleArr, "data", data.data(), data.size() * 8);
    put_int(o, "SubWidth", width);
    put_int(o, "SubHeight", height);
    put_int(o, "OffsetX", 0);
    put_int(o, "OffsetY", 0);
    put_section(o, kBsEndaStream, "", nullptr, 0);
    FILE* f = std::fopen(path, "wb");
    if (!f) return B2M_ERR_ARG;
    const size_t put = std::fwrite(o.data(), 1, o.size(), f);
    const int closed = std::fclose(f);
    return (put == o.size() && closed == 0) ? B2M_OK : B2M_ERR_ARG;
}
