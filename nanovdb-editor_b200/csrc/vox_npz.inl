// vox_npz.inl - raster_file and create_gaussian_data_from_arrays
// (raster/RasterUtils.cpp:208-395), included by vox_dropin.cu.
//
// raster_file reads the Gaussian arrays the reference looks up by name
// (means, opacities, quaternions, scales, sh_0, sh_n; RasterUtils.cpp:322-325)
// from an .npz archive or a .ply file, the two formats the reference's
// fileformat module loads for it (fileformat/FileFormat.cpp:51, :766-790).
// .npz: the layout numpy.savez writes - stored (uncompressed) zip entries,
// ZIP64 sizes allowed, each entry a little-endian float32 C-order .npy array.
// .ply: the binary Gaussian-splat layout FileFormat.cpp:205-580 reads - vertex
// properties as 4-byte floats (little or big endian), x/y/z -> means,
// opacity, rot_0..3 -> quaternions, scale_0..2 -> scales, f_dc_0..2 -> sh_0,
// 45 f_rest_* -> sh_n, red/green/blue -> colors.  Unlike the reference, header
// lines may end in CRLF, and a vertex property that is not a 4-byte float is
// rejected rather than misread.  Other formats (e57, ingp, compressed npz)
// are reported as unsupported.

namespace
{

struct NpzArray
{
    std::string name;
    std::vector<float> data;
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

// parses one .npy payload; float32 little-endian, C order only
static bool parse_npy(const unsigned char* p, uint64_t size, std::vector<float>& out)
{
    if (size < 10 || memcmp(p, "\x93NUMPY", 6) != 0)
        return false;
    uint8_t major = p[6];
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
    if (hoff + hlen > size)
        return false;
    std::string hdr((const char*)p + hoff, (size_t)hlen);
    if (hdr.find("'<f4'") == std::string::npos && hdr.find("'float32'") == std::string::npos)
        return false;
    if (hdr.find("'fortran_order': True") != std::string::npos)
        return false;
    size_t sp = hdr.find("'shape':");
    if (sp == std::string::npos)
        return false;
    size_t lp = hdr.find('(', sp), rp = hdr.find(')', sp);
    if (lp == std::string::npos || rp == std::string::npos)
        return false;
    uint64_t count = 1;
    std::string dims = hdr.substr(lp + 1, rp - lp - 1);
    bool any = false;
    size_t i = 0;
    while (i < dims.size())
    {
        while (i < dims.size() && (dims[i] < '0' || dims[i] > '9'))
            i++;
        if (i >= dims.size())
            break;
        uint64_t v = 0;
        while (i < dims.size() && dims[i] >= '0' && dims[i] <= '9')
            v = v * 10 + (uint64_t)(dims[i++] - '0');
        count *= v;
        any = true;
    }
    if (!any)
        count = 1;
    uint64_t data_off = hoff + hlen;
    if (data_off + count * 4 > size)
        return false;
    out.resize((size_t)count);
    if (count)
        memcpy(out.data(), p + data_off, (size_t)count * 4);
    return true;
}

static bool read_npz(const char* path, std::vector<NpzArray>& arrays, std::string& why)
{
    FILE* f = fopen(path, "rb");
    if (!f)
    {
        why = "cannot open file";
        return false;
    }
    std::vector<unsigned char> buf;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (n > 0)
    {
        buf.resize((size_t)n);
        if (fread(buf.data(), 1, (size_t)n, f) != (size_t)n)
            buf.clear();
    }
    fclose(f);
    uint64_t pos = 0, total = buf.size();
    while (pos + 30 <= total && rd32(&buf[pos]) == 0x04034b50u)
    {
        const unsigned char* h = &buf[pos];
        uint16_t method = rd16(h + 8);
        uint64_t csize = rd32(h + 18), usize = rd32(h + 22);
        uint16_t nlen = rd16(h + 26), xlen = rd16(h + 28);
        if (pos + 30 + nlen + xlen > total)
            break;
        std::string name((const char*)h + 30, nlen);
        const unsigned char* x = h + 30 + nlen;
        for (uint32_t xo = 0; xo + 4 <= xlen;)
        {
            uint16_t id = rd16(x + xo), len = rd16(x + xo + 2);
            if (id == 0x0001 && len >= 16)
            {
                usize = rd64(x + xo + 4);
                csize = rd64(x + xo + 12);
            }
            xo += 4u + len;
        }
        uint64_t data = pos + 30 + nlen + xlen;
        if (method != 0)
        {
            why = "compressed npz entries are not supported (save with numpy.savez)";
            return false;
        }
        if (data + csize > total || csize != usize)
        {
            why = "truncated npz entry";
            return false;
        }
        if (name.size() > 4 && name.compare(name.size() - 4, 4, ".npy") == 0)
            name.resize(name.size() - 4);
        NpzArray a;
        a.name = name;
        if (!parse_npy(&buf[data], csize, a.data))
        {
            why = "entry '" + name + "' is not a little-endian float32 C-order array";
            return false;
        }
        arrays.push_back(std::move(a));
        pos = data + csize;
    }
    if (arrays.empty())
    {
        why = "no npz entries found";
        return false;
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

static bool read_ply(const char* path, std::vector<NpzArray>& arrays, std::string& why)
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
                vertex_count = (uint64_t)strtoull(line.c_str() + 15, nullptr, 10);
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
    if (bad_prop)
    {
        fclose(f);
        why = "every vertex property must be a 4-byte float";
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
    const size_t nprop = props.size();
    std::vector<float> rows(nprop * (size_t)vertex_count);
    const size_t got = nprop ? fread(rows.data(), sizeof(float) * nprop, (size_t)vertex_count, f) : 0;
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
        a.data.resize((size_t)vertex_count * ncol);
        for (uint64_t v = 0; v < vertex_count; v++)
            for (int c = 0; c < ncol; c++)
                a.data[(size_t)v * ncol + c] = rows[(size_t)v * nprop + cols[c]];
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

} // namespace

static pnanovdb_bool_t PNANOVDB_ABI r_create_from_arrays(pnanovdb_raster_t* raster, const pnanovdb_compute_t*,
                                                         pnanovdb_compute_queue_t* queue,
                                                         pnanovdb_compute_array_t** arrays, pnanovdb_uint32_t count,
                                                         pnanovdb_raster_gaussian_data_t** gaussian_data,
                                                         pnanovdb_raster_shader_params_t*,
                                                         pnanovdb_raster_context_t** raster_context)
{
    if (!arrays || count < 5u || !gaussian_data)
        return PNANOVDB_FALSE;
    pnanovdb_compute_array_t *m = arrays[0], *o = arrays[1], *q = arrays[2], *s = arrays[3], *c = arrays[4];
    if (!m || m->element_size != 4)
        return PNANOVDB_FALSE;
    pnanovdb_raster_gaussian_data_t* d = new pnanovdb_raster_gaussian_data_t();
    d->n = (int64_t)(m->element_count / 3);
    d->device = queue_device(queue);
    d->raw = 1;
    if (!(copy_floats(d->means, m, 3 * d->n) && copy_floats(d->opacities, o, d->n) &&
          copy_floats(d->quats, q, 4 * d->n) && copy_floats(d->scales, s, 3 * d->n) &&
          copy_floats(d->colors, c, 3 * d->n)))
    {
        log_err("create_gaussian_data_from_arrays: arrays must be float32 [means, opacities, quaternions, scales, sh_0]");
        delete d;
        return PNANOVDB_FALSE;
    }
    *gaussian_data = d;
    if (raster_context && !*raster_context)
    {
        *raster_context = r_create_context(raster ? raster->compute : nullptr, queue);
        if (!*raster_context)
        {
            delete d;
            *gaussian_data = nullptr;
            return PNANOVDB_FALSE;
        }
    }
    return PNANOVDB_TRUE;
}

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
    std::vector<NpzArray> arrays;
    std::string why;
    bool loaded = false;
    if (has_suffix(filename, ".ply"))
        loaded = read_ply(filename, arrays, why);
    else if (has_suffix(filename, ".npz"))
        loaded = read_npz(filename, arrays, why);
    else
        why = "file format not supported (.npz and .ply are)";
    if (!loaded)
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
    int64_t n = (int64_t)(ca[0]->element_count / 3);
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
    *nanovdb_arr = run_host(queue_device(queue), &g, voxel_size, cull_from_params(shader_params_arrays),
                            VOX_FLAG_RAW_INPUTS | DROPIN_ORDER, profiler_report, userdata);
    return *nanovdb_arr ? PNANOVDB_TRUE : PNANOVDB_FALSE;
}
