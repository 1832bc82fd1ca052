// vox_npz.inl - raster_file and create_gaussian_data_from_arrays
// (raster/RasterUtils.cpp:208-395), included by vox_dropin.cu.
//
// raster_file reads the Gaussian arrays the reference looks up by name
// (means, opacities, quaternions, scales, sh_0, sh_n; RasterUtils.cpp:322-325)
// from an .npz archive or a .ply file, the two formats the reference's
// fileformat module loads for it (fileformat/FileFormat.cpp:51, :766-790).
// .npz: a zip archive as numpy.savez (stored) or numpy.savez_compressed
// (deflated) writes it, ZIP64 records allowed, each entry a little-endian
// float32 C-order .npy array; an "sh" array of shape (G, K, 3) stands for
// sh_0 / sh_n as in FileFormat.cpp:113-188.
// .ply: the binary Gaussian-splat layout FileFormat.cpp:205-580 reads - vertex
// properties as 4-byte floats (little or big endian), x/y/z -> means,
// opacity, rot_0..3 -> quaternions, scale_0..2 -> scales, f_dc_0..2 -> sh_0,
// 45 f_rest_* -> sh_n, red/green/blue -> colors.  Unlike the reference, header
// lines may end in CRLF, and a vertex property that is not a 4-byte float is
// rejected rather than misread.  Other formats (e57, ingp) are reported as
// unsupported.
//
// Every size and count in a file is untrusted: each is checked against the
// bytes actually present (with overflow-checked arithmetic) before anything is
// allocated or read, and allocation failures are reported as errors, so a
// malformed file can neither overrun a buffer nor throw across the C ABI.

#include <cerrno>
#include <climits>
#include <new>
#include <zlib.h>

namespace
{

// Host float storage of one parsed array: page-locked (from the pool of
// pinned_alloc, so the upload that follows runs at link speed) or, when that
// is not asked for or not available, ordinary heap memory.
class FloatBuf
{
  public:
    FloatBuf() = default;
    FloatBuf(const FloatBuf&) = delete;
    FloatBuf& operator=(const FloatBuf&) = delete;
    FloatBuf(FloatBuf&& o) noexcept : p_(o.p_), n_(o.n_), pinned_(o.pinned_)
    {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    FloatBuf& operator=(FloatBuf&& o) noexcept
    {
        if (this != &o)
        {
            reset();
            p_ = o.p_;
            n_ = o.n_;
            pinned_ = o.pinned_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    ~FloatBuf()
    {
        reset();
    }
    // count floats, uninitialised; throws std::bad_alloc when memory runs out
    void resize(size_t count, bool want_pinned)
    {
        reset();
        const size_t bytes = count * sizeof(float) + 16;
        p_ = want_pinned ? (float*)pinned_alloc(bytes) : nullptr;
        pinned_ = p_ != nullptr;
        if (!p_)
            p_ = (float*)malloc(bytes);
        if (!p_)
            throw std::bad_alloc();
        n_ = count;
    }
    float* data()
    {
        return p_;
    }
    const float* data() const
    {
        return p_;
    }
    size_t size() const
    {
        return n_;
    }
    // hands the storage to a compute array (freed by array_destroy)
    pnanovdb_compute_array_t* release_to_array()
    {
        pnanovdb_compute_array_t* a = (pnanovdb_compute_array_t*)calloc(1, sizeof(pnanovdb_compute_array_t));
        if (!a)
            return nullptr;
        a->data = p_;
        a->element_size = 4;
        a->element_count = n_;
        p_ = nullptr;
        n_ = 0;
        return a;
    }

  private:
    void reset()
    {
        if (p_ && !(pinned_ && pinned_release(p_)))
            free(p_);
        p_ = nullptr;
        n_ = 0;
    }
    float* p_ = nullptr;
    size_t n_ = 0;
    bool pinned_ = false;
};

struct NpzArray
{
    std::string name;
    FloatBuf data;
    std::vector<uint64_t> shape;
};

static uint16_t rd16(const unsigned char* p)
{
    return (uint16_t)(p[0] | (p[1] << 8));
}
static uint32_t rd32(const unsigned char* p)
{
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint64_t rd64(const unsigned char* p)
{
    return (uint64_t)rd32(p) | ((uint64_t)rd32(p + 4) << 32);
}

// a * b without wrapping; false when the product does not fit in 64 bits
static bool mul_u64(uint64_t a, uint64_t b, uint64_t& r)
{
    if (a && b > UINT64_MAX / a)
        return false;
    r = a * b;
    return true;
}

// Parses one .npy payload of `size` bytes: float32 little-endian, C order.
// Every count comes from the payload, so each is checked against its size
// before anything is allocated or copied.
static bool parse_npy(const unsigned char* p, uint64_t size, NpzArray& out, bool pinned)
{
    if (size < 10 || memcmp(p, "\x93NUMPY", 6) != 0)
        return false;
    const uint8_t major = p[6];
    uint64_t hlen, hoff;
    if (major == 1)
    {
        hlen = rd16(p + 8);
        hoff = 10;
    }
    else
    {
        if (size < 12)
            return false;
        hlen = rd32(p + 8);
        hoff = 12;
    }
    if (hlen > size - hoff)
        return false;
    std::string hdr((const char*)p + hoff, (size_t)hlen);
    if (hdr.find("'<f4'") == std::string::npos && hdr.find("'float32'") == std::string::npos)
        return false;
    if (hdr.find("'fortran_order': True") != std::string::npos)
        return false;
    const size_t sp = hdr.find("'shape':");
    if (sp == std::string::npos)
        return false;
    const size_t lp = hdr.find('(', sp), rp = hdr.find(')', sp);
    if (lp == std::string::npos || rp == std::string::npos || rp < lp)
        return false;
    uint64_t count = 1;
    const std::string dims = hdr.substr(lp + 1, rp - lp - 1);
    out.shape.clear();
    size_t i = 0;
    while (i < dims.size())
    {
        while (i < dims.size() && (dims[i] < '0' || dims[i] > '9'))
            i++;
        if (i >= dims.size())
            break;
        uint64_t v = 0;
        while (i < dims.size() && dims[i] >= '0' && dims[i] <= '9')
        {
            if (v > (UINT64_MAX - 9) / 10)
                return false;
            v = v * 10 + (uint64_t)(dims[i++] - '0');
        }
        if (!mul_u64(count, v, count))
            return false;
        out.shape.push_back(v);
    }
    const uint64_t data_off = hoff + hlen;
    if (count > (size - data_off) / 4)
        return false;
    out.data.resize((size_t)count, pinned);
    if (count)
        memcpy(out.data.data(), p + data_off, (size_t)count * 4);
    return true;
}

static bool read_file(const char* path, std::vector<unsigned char>& buf, std::string& why)
{
    FILE* f = fopen(path, "rb");
    if (!f)
    {
        why = "cannot open file";
        return false;
    }
    bool ok = fseek(f, 0, SEEK_END) == 0;
    const long n = ok ? ftell(f) : -1;
    ok = ok && n >= 0 && fseek(f, 0, SEEK_SET) == 0;
    if (ok && n > 0)
    {
        buf.resize((size_t)n);
        ok = fread(buf.data(), 1, (size_t)n, f) == (size_t)n;
    }
    fclose(f);
    if (!ok)
        why = "cannot read file";
    return ok;
}

// Inflates a raw deflate stream (zip method 8) of exactly `usize` bytes.
static bool inflate_raw(const unsigned char* src, uint64_t csize, uint64_t usize, std::vector<unsigned char>& dst)
{
    // deflate expands at most about 1032:1; a larger claimed size is corrupt
    uint64_t lim;
    if (!mul_u64(csize, 1040, lim) || usize > lim + 1024)
        return false;
    dst.resize((size_t)usize);
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit2(&zs, -MAX_WBITS) != Z_OK)
        return false;
    uint64_t in_done = 0, out_done = 0;
    int rc = Z_OK;
    while (rc == Z_OK)
    {
        const uint64_t in_left = csize - in_done, out_left = usize - out_done;
        zs.next_in = const_cast<unsigned char*>(src + in_done);
        zs.avail_in = (uInt)(in_left < (1u << 30) ? in_left : (1u << 30));
        zs.next_out = dst.data() + out_done;
        zs.avail_out = (uInt)(out_left < (1u << 30) ? out_left : (1u << 30));
        const uInt ai = zs.avail_in, ao = zs.avail_out;
        rc = inflate(&zs, Z_NO_FLUSH);
        in_done += ai - zs.avail_in;
        out_done += ao - zs.avail_out;
        if (rc == Z_BUF_ERROR && (ai == zs.avail_in && ao == zs.avail_out))
            break; // no progress: truncated stream or more output than claimed
        if (rc == Z_BUF_ERROR)
            rc = Z_OK;
    }
    inflateEnd(&zs);
    return rc == Z_STREAM_END && out_done == usize;
}

// .npz: a zip archive of .npy entries (numpy.savez stores them, numpy.savez_compressed
// deflates them; cnpy reads both, fileformat/FileFormat.cpp:87-112).  Entries are found
// through the central directory (ZIP64 records included); each local header is then
// read for the name / extra lengths, and every offset and size is checked against the
// file before use.  The CRC-32 of each entry is verified.
static bool read_npz(const char* path, std::vector<NpzArray>& arrays, std::string& why, bool pinned)
{
    std::vector<unsigned char> buf;
    if (!read_file(path, buf, why))
        return false;
    const uint64_t total = buf.size();
    const unsigned char* b = buf.data();
    // end of central directory: 22 bytes plus a comment of at most 65535
    uint64_t eocd = UINT64_MAX;
    for (uint64_t back = 22; back <= total && back <= 22 + 65535; back++)
        if (rd32(b + total - back) == 0x06054b50u)
        {
            eocd = total - back;
            break;
        }
    if (eocd == UINT64_MAX)
    {
        why = "not a zip archive (no end of central directory)";
        return false;
    }
    uint64_t n_entries = rd16(b + eocd + 10), cd_size = rd32(b + eocd + 12), cd_off = rd32(b + eocd + 16);
    if ((n_entries == 0xFFFFu || cd_size == 0xFFFFFFFFu || cd_off == 0xFFFFFFFFu) && eocd >= 20 &&
        rd32(b + eocd - 20) == 0x07064b50u)
    {
        const uint64_t z64 = rd64(b + eocd - 20 + 8); // ZIP64 end of central directory record
        if (z64 > total || total - z64 < 56 || rd32(b + z64) != 0x06064b50u)
        {
            why = "corrupt ZIP64 end of central directory";
            return false;
        }
        n_entries = rd64(b + z64 + 32);
        cd_size = rd64(b + z64 + 40);
        cd_off = rd64(b + z64 + 48);
    }
    if (cd_off > total || cd_size > total - cd_off)
    {
        why = "corrupt zip central directory";
        return false;
    }
    uint64_t pos = cd_off;
    const uint64_t cd_end = cd_off + cd_size;
    for (uint64_t e = 0; e < n_entries; e++)
    {
        if (cd_end - pos < 46 || rd32(b + pos) != 0x02014b50u)
        {
            why = "corrupt zip central directory entry";
            return false;
        }
        const unsigned char* h = b + pos;
        const uint16_t method = rd16(h + 10);
        const uint32_t crc = rd32(h + 16);
        uint64_t csize = rd32(h + 20), usize = rd32(h + 24);
        const uint16_t nlen = rd16(h + 28), xlen = rd16(h + 30), clen = rd16(h + 32);
        uint64_t lho = rd32(h + 42);
        if ((uint64_t)46 + nlen + xlen + clen > cd_end - pos)
        {
            why = "corrupt zip central directory entry";
            return false;
        }
        std::string name((const char*)h + 46, nlen);
        // ZIP64 extended information: the 64-bit values of the fields set to all ones, in order
        const unsigned char* x = h + 46 + nlen;
        for (uint32_t xo = 0; xo + 4 <= xlen;)
        {
            const uint16_t id = rd16(x + xo), len = rd16(x + xo + 2);
            if ((uint32_t)xo + 4u + len > xlen)
                break;
            if (id == 0x0001)
            {
                uint32_t f = xo + 4;
                const uint32_t fe = xo + 4 + len;
                if (usize == 0xFFFFFFFFu && f + 8 <= fe)
                {
                    usize = rd64(x + f);
                    f += 8;
                }
                if (csize == 0xFFFFFFFFu && f + 8 <= fe)
                {
                    csize = rd64(x + f);
                    f += 8;
                }
                if (lho == 0xFFFFFFFFu && f + 8 <= fe)
                    lho = rd64(x + f);
            }
            xo += 4u + len;
        }
        pos += (uint64_t)46 + nlen + xlen + clen;
        if (lho > total || total - lho < 30 || rd32(b + lho) != 0x04034b50u)
        {
            why = "corrupt zip local header";
            return false;
        }
        const uint64_t data = lho + 30 + rd16(b + lho + 26) + rd16(b + lho + 28);
        if (data > total || csize > total - data)
        {
            why = "truncated npz entry";
            return false;
        }
        const unsigned char* payload = b + data;
        std::vector<unsigned char> inflated;
        if (method == 8)
        {
            if (!inflate_raw(payload, csize, usize, inflated))
            {
                why = "corrupt deflate stream in npz entry '" + name + "'";
                return false;
            }
            payload = inflated.data();
        }
        else if (method != 0 || csize != usize)
        {
            why = "npz entry '" + name + "' uses an unsupported zip compression method";
            return false;
        }
        uint64_t done = 0;
        uLong c = crc32(0L, Z_NULL, 0);
        while (done < usize)
        {
            const uint64_t step = usize - done < (1u << 30) ? usize - done : (1u << 30);
            c = crc32(c, payload + done, (uInt)step);
            done += step;
        }
        if ((uint32_t)c != crc)
        {
            why = "CRC mismatch in npz entry '" + name + "'";
            return false;
        }
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".npy") == 0)
            name.resize(name.size() - 4);
        NpzArray a;
        a.name = name;
        if (!parse_npy(payload, usize, a, pinned))
        {
            why = "entry '" + name + "' is not a little-endian float32 C-order array";
            return false;
        }
        arrays.push_back(std::move(a));
    }
    if (arrays.empty())
    {
        why = "no npz entries found";
        return false;
    }
    // the "sh" alias (fileformat/FileFormat.cpp:113-188): an array of shape
    // (G, K, W) stands for sh_0 = sh[:, 0, :] and sh_n = sh[:, 1:, :]
    bool has0 = false, hasn = false;
    const NpzArray* sh = nullptr;
    for (const auto& a : arrays)
    {
        has0 = has0 || a.name == "sh_0";
        hasn = hasn || a.name == "sh_n";
        if (a.name == "sh")
            sh = &a;
    }
    if (sh && (!has0 || !hasn) && sh->shape.size() >= 2 && sh->shape[1] >= 1)
    {
        const uint64_t stride = sh->shape[1], width = sh->shape.size() >= 3 ? sh->shape[2] : 1;
        const uint64_t rows = sh->data.size() / (stride * width);
        NpzArray s0, sn;
        s0.name = "sh_0";
        sn.name = "sh_n";
        s0.data.resize((size_t)(rows * width), pinned);
        sn.data.resize((size_t)(rows * (stride - 1) * width), pinned);
        for (uint64_t r = 0; r < rows; r++)
        {
            const float* src = sh->data.data() + r * stride * width;
            memcpy(s0.data.data() + r * width, src, (size_t)width * 4);
            if (stride > 1)
                memcpy(sn.data.data() + r * (stride - 1) * width, src + width, (size_t)((stride - 1) * width) * 4);
        }
        if (!has0)
            arrays.push_back(std::move(s0));
        if (!hasn)
            arrays.push_back(std::move(sn));
    }
    return true;
}

// one header line without its line ending (LF or CRLF)
static std::string ply_line(const std::string& raw)
{
    std::string l = raw;
    while (!l.empty() && (l.back() == '\n' || l.back() == '\r'))
        l.pop_back();
    return l;
}

static bool read_ply(const char* path, std::vector<NpzArray>& arrays, std::string& why, bool pinned)
{
    FILE* f = fopen(path, "rb");
    if (!f)
    {
        why = "cannot open file";
        return false;
    }
    std::vector<std::string> props; // vertex property names, in file order
    uint64_t vertex_count = 0;
    bool in_vertex = false, big_endian = false, binary = false, header_done = false, bad_prop = false;
    bool bad_count = false;
    char buf[512];
    while (fgets(buf, sizeof(buf), f))
    {
        const std::string line = ply_line(buf);
        if (line == "end_header")
        {
            header_done = true;
            break;
        }
        if (line.rfind("format ", 0) == 0)
        {
            binary = line.find("binary_little_endian") != std::string::npos ||
                     line.find("binary_big_endian") != std::string::npos;
            big_endian = line.find("binary_big_endian") != std::string::npos;
        }
        else if (line.rfind("element ", 0) == 0)
        {
            in_vertex = line.rfind("element vertex ", 0) == 0;
            if (in_vertex)
            {
                const char* s = line.c_str() + 15;
                char* end = nullptr;
                errno = 0;
                vertex_count = (uint64_t)strtoull(s, &end, 10);
                bad_count = end == s || errno == ERANGE || *s == '-';
            }
        }
        else if (line.rfind("property ", 0) == 0 && in_vertex)
        {
            const size_t sp = line.find(' ', 9);
            const std::string type = line.substr(9, sp == std::string::npos ? std::string::npos : sp - 9);
            if (type != "float" && type != "float32")
                bad_prop = true;
            props.push_back(sp == std::string::npos ? std::string() : line.substr(sp + 1));
        }
    }
    if (!header_done || !binary)
    {
        fclose(f);
        why = header_done ? "only binary ply files are supported" : "no ply header";
        return false;
    }
    if (bad_prop || props.empty() || bad_count)
    {
        fclose(f);
        why = bad_count ? "bad vertex count in the ply header"
                        : "every vertex property must be a 4-byte float (and there must be one)";
        return false;
    }
    // the vertex count comes from the file: bound it by the bytes that follow the header
    const long here = ftell(f);
    const bool sized = here >= 0 && fseek(f, 0, SEEK_END) == 0;
    const long end = sized ? ftell(f) : -1;
    if (!sized || end < here || fseek(f, here, SEEK_SET) != 0)
    {
        fclose(f);
        why = "cannot read file";
        return false;
    }
    const size_t nprop = props.size();
    const uint64_t row_bytes = 4 * (uint64_t)nprop;
    if (vertex_count > (uint64_t)(end - here) / row_bytes)
    {
        fclose(f);
        why = "truncated ply vertex data";
        return false;
    }
    auto col = [&](const char* name) -> int {
        for (size_t i = 0; i < props.size(); i++)
            if (props[i] == name)
                return (int)i;
        return -1;
    };
    const int x = col("x"), y = col("y"), z = col("z"), op = col("opacity");
    const int r[4] = { col("rot_0"), col("rot_1"), col("rot_2"), col("rot_3") };
    const int sc[3] = { col("scale_0"), col("scale_1"), col("scale_2") };
    const int dc[3] = { col("f_dc_0"), col("f_dc_1"), col("f_dc_2") };
    const int rest0 = col("f_rest_0");
    const int rgb[3] = { col("red"), col("green"), col("blue") };
    std::vector<float> rows(nprop * (size_t)vertex_count);
    const size_t got = vertex_count ? fread(rows.data(), (size_t)row_bytes, (size_t)vertex_count, f) : 0;
    fclose(f);
    if (got != (size_t)vertex_count)
    {
        why = "truncated ply vertex data";
        return false;
    }
    if (big_endian)
        for (float& v : rows)
        {
            uint32_t u;
            memcpy(&u, &v, 4);
            u = (u >> 24) | ((u >> 8) & 0xFF00u) | ((u << 8) & 0xFF0000u) | (u << 24);
            memcpy(&v, &u, 4);
        }
    auto gather = [&](const char* name, const int* cols, int ncol) {
        for (int c = 0; c < ncol; c++)
            if (cols[c] < 0)
                return;
        NpzArray a;
        a.name = name;
        a.data.resize((size_t)vertex_count * ncol, pinned);
        for (uint64_t v = 0; v < vertex_count; v++)
            for (int c = 0; c < ncol; c++)
                a.data.data()[(size_t)v * ncol + c] = rows[(size_t)v * nprop + cols[c]];
        arrays.push_back(std::move(a));
    };
    const int xyz[3] = { x, y, z };
    gather("means", xyz, 3);
    gather("opacities", &op, 1);
    gather("quaternions", r, 4);
    gather("scales", sc, 3);
    gather("sh_0", dc, 3);
    gather("colors", rgb, 3);
    if (rest0 >= 0 && rest0 + 45 <= (int)nprop)
    {
        int rest[45];
        for (int i = 0; i < 45; i++)
            rest[i] = rest0 + i;
        gather("sh_n", rest, 45);
    }
    return true;
}

// Loads the Gaussian arrays of a .npz / .ply file (into page-locked memory when
// `pinned`); false with a reason on any malformed input or when memory runs out
// (nothing throws past this point).
static bool read_gaussian_file(const char* path, std::vector<NpzArray>& arrays, std::string& why, bool pinned);

static bool has_suffix(const char* s, const char* suffix)
{
    const size_t n = strlen(s), m = strlen(suffix);
    if (n < m)
        return false;
    for (size_t i = 0; i < m; i++)
        if (tolower((unsigned char)s[n - m + i]) != suffix[i])
            return false;
    return true;
}

static bool read_gaussian_file(const char* path, std::vector<NpzArray>& arrays, std::string& why, bool pinned)
{
    try
    {
        if (has_suffix(path, ".ply"))
            return read_ply(path, arrays, why, pinned);
        if (has_suffix(path, ".npz"))
            return read_npz(path, arrays, why, pinned);
        why = "file format not supported (.npz and .ply are)";
    }
    catch (const std::bad_alloc&)
    {
        arrays.clear();
        why = "out of host memory";
    }
    catch (const std::exception& e)
    {
        arrays.clear();
        why = e.what();
    }
    return false;
}

} // namespace

// raster/RasterUtils.cpp:208-245: arrays in the on-disk convention (log-scales,
// logit opacities, SH0) -> gaussian data (+ a raster context when asked)
static pnanovdb_bool_t PNANOVDB_ABI r_create_from_arrays(pnanovdb_raster_t* raster, const pnanovdb_compute_t*,
                                                         pnanovdb_compute_queue_t* queue,
                                                         pnanovdb_compute_array_t** arrays, pnanovdb_uint32_t count,
                                                         pnanovdb_raster_gaussian_data_t** gaussian_data,
                                                         pnanovdb_raster_shader_params_t*,
                                                         pnanovdb_raster_context_t** raster_context)
{
    if (!arrays || count < 5u || !gaussian_data)
        return PNANOVDB_FALSE;
    return no_throw<pnanovdb_bool_t>("create_gaussian_data_from_arrays", PNANOVDB_FALSE, [&]() -> pnanovdb_bool_t {
        pnanovdb_compute_array_t *m = arrays[0], *o = arrays[1], *q = arrays[2], *s = arrays[3], *c = arrays[4];
        if (!m || m->element_size != 4)
        {
            log_err("create_gaussian_data_from_arrays: means must be float32");
            return PNANOVDB_FALSE;
        }
        std::unique_ptr<pnanovdb_raster_gaussian_data_t> d(new pnanovdb_raster_gaussian_data_t());
        d->n = (int64_t)(m->element_count / 3);
        d->device = queue_device(queue);
        d->raw = 1;
        if (!(copy_floats(d->means, m, 3 * d->n) && copy_floats(d->opacities, o, d->n) &&
              copy_floats(d->quats, q, 4 * d->n) && copy_floats(d->scales, s, 3 * d->n) &&
              copy_floats(d->colors, c, 3 * d->n)))
        {
            log_err("create_gaussian_data_from_arrays: arrays must be float32 [means, opacities, quaternions, scales, sh_0]");
            return PNANOVDB_FALSE;
        }
        if (raster_context && !*raster_context)
        {
            *raster_context = r_create_context(raster ? raster->compute : nullptr, queue);
            if (!*raster_context)
                return PNANOVDB_FALSE;
        }
        *gaussian_data = d.release();
        return PNANOVDB_TRUE;
    });
}

// raster/RasterUtils.cpp:247-398: a .npz / .ply file -> the node2 grid with its
// RGBA8 values, or (with gaussian_data and raster_context) the gaussian data
static pnanovdb_bool_t PNANOVDB_ABI r_raster_file(pnanovdb_raster_t* raster, const pnanovdb_compute_t* compute,
                                                  pnanovdb_compute_queue_t* queue, const char* filename,
                                                  float voxel_size, pnanovdb_compute_array_t** nanovdb_arr,
                                                  pnanovdb_raster_gaussian_data_t** gaussian_data,
                                                  pnanovdb_raster_context_t** raster_context,
                                                  pnanovdb_compute_array_t** shader_params_arrays,
                                                  pnanovdb_raster_shader_params_t* raster_params,
                                                  pnanovdb_profiler_report_t profiler_report, void* userdata)
{
    if (!filename)
        return PNANOVDB_FALSE;
    return no_throw<pnanovdb_bool_t>("raster_file", PNANOVDB_FALSE, [&]() -> pnanovdb_bool_t {
        std::vector<NpzArray> arrays;
        std::string why;
        if (!read_gaussian_file(filename, arrays, why, true))
        {
            std::string msg = std::string("raster_file: failed to load Gaussian data from '") + filename + "': " + why;
            log_err(msg.c_str());
            return PNANOVDB_FALSE;
        }
        const char* names[6] = { "means", "opacities", "quaternions", "scales", "sh_0", "sh_n" };
        pnanovdb_compute_array_t* ca[6] = {};
        pnanovdb_compute_array_t holder[6] = {};
        for (int i = 0; i < 6; i++)
        {
            for (auto& a : arrays)
                if (a.name == names[i])
                {
                    holder[i].data = a.data.data();
                    holder[i].element_size = 4;
                    holder[i].element_count = a.data.size();
                    ca[i] = &holder[i];
                }
            if (i < 5 && !ca[i])
            {
                std::string msg = std::string("raster_file: '") + filename + "' has no array '" + names[i] + "'";
                log_err(msg.c_str());
                return PNANOVDB_FALSE;
            }
        }
        if (gaussian_data && raster_context)
        {
            pnanovdb_bool_t ok = r_create_from_arrays(raster, compute, queue, ca, 6, gaussian_data, raster_params,
                                                      raster_context);
            if (ok && *gaussian_data)
                (*gaussian_data)->cull_scale = cull_from_params(shader_params_arrays);
            return ok;
        }
        if (!nanovdb_arr)
            return PNANOVDB_FALSE;
        const int64_t n = (int64_t)(ca[0]->element_count / 3);
        if ((int64_t)ca[1]->element_count < n || (int64_t)ca[2]->element_count < 4 * n ||
            (int64_t)ca[3]->element_count < 3 * n || (int64_t)ca[4]->element_count < 3 * n)
        {
            log_err("raster_file: attribute counts do not match means");
            return PNANOVDB_FALSE;
        }
        vox_gaussians_t g;
        g.count = n;
        g.means = (const float*)ca[0]->data;
        g.opacities = (const float*)ca[1]->data;
        g.quats = (const float*)ca[2]->data;
        g.scales = (const float*)ca[3]->data;
        g.colors = (const float*)ca[4]->data;
        *nanovdb_arr = run_host(queue, &g, voxel_size, cull_from_params(shader_params_arrays),
                                VOX_FLAG_RAW_INPUTS | DROPIN_ORDER, profiler_report, userdata, "raster_file");
        return *nanovdb_arr ? PNANOVDB_TRUE : PNANOVDB_FALSE;
    });
}

// fileformat/FileFormat.cpp:68-80: the extensions load_file accepts
static pnanovdb_bool_t PNANOVDB_ABI ff_can_load_file(const char* filename)
{
    return filename && (has_suffix(filename, ".npz") || has_suffix(filename, ".ply")) ? PNANOVDB_TRUE : PNANOVDB_FALSE;
}

// fileformat/FileFormat.cpp:754-800: every named array, or FALSE (and no
// arrays) when the file cannot be read or lacks one of them
static pnanovdb_bool_t PNANOVDB_ABI ff_load_file(const char* filename, pnanovdb_uint32_t array_count,
                                                 const char** array_names, pnanovdb_compute_array_t** out_arrays)
{
    if (!filename || !array_names || !out_arrays)
        return PNANOVDB_FALSE;
    return no_throw<pnanovdb_bool_t>("load_file", PNANOVDB_FALSE, [&]() -> pnanovdb_bool_t {
        for (pnanovdb_uint32_t i = 0; i < array_count; i++)
            out_arrays[i] = nullptr;
        std::vector<NpzArray> arrays;
        std::string why;
        if (!read_gaussian_file(filename, arrays, why, false))
        {
            log_err((std::string("load_file: failed to load '") + filename + "': " + why).c_str());
            return PNANOVDB_FALSE;
        }
        std::vector<NpzArray*> pick(array_count, nullptr);
        for (pnanovdb_uint32_t i = 0; i < array_count; i++)
        {
            for (auto& a : arrays)
                if (array_names[i] && a.name == array_names[i])
                    pick[i] = &a;
            if (!pick[i])
            {
                log_err((std::string("load_file: '") + filename + "' has no array '" +
                         (array_names[i] ? array_names[i] : "(null)") + "'")
                            .c_str());
                return PNANOVDB_FALSE;
            }
        }
        for (pnanovdb_uint32_t i = 0; i < array_count; i++)
        {
            // a name asked for twice gets its own copy
            bool dup = false;
            for (pnanovdb_uint32_t k = 0; k < i; k++)
                dup = dup || pick[k] == pick[i];
            out_arrays[i] = dup ? array_create(4, pick[i]->data.size(), pick[i]->data.data())
                                : pick[i]->data.release_to_array();
            if (!out_arrays[i])
            {
                for (pnanovdb_uint32_t k = 0; k < i; k++)
                {
                    array_destroy(out_arrays[k]);
                    out_arrays[k] = nullptr;
                }
                log_err("load_file: out of host memory");
                return PNANOVDB_FALSE;
            }
        }
        return PNANOVDB_TRUE;
    });
}
