// output.cpp -- trajectory (XML, PDB) and RDF (CSV) files of the standalone
// native harness, in the formats of the reference's outputHandler
// (lib/ReaDDyGPU_Cpp/outputHandler/outputHandler.cpp); see
// include/readdy_b200_output.h for what differs and why.
#include "readdy_b200_output.h"

#include <cstdio>
#include <string>

struct rdgpu_traj {
    FILE* f = nullptr;
    int32_t format = RDGPU_TRAJ_XML;
    std::string path;
};

namespace {

thread_local std::string g_out_err;

int out_fail(const std::string& msg, int code = RDGPU_ERR_ARG)
{
    g_out_err = msg;
    return code;
}

// %.17g round-trips every double; shortest-form printing is not needed here
void put_coord(FILE* f, double v) { std::fprintf(f, "%.17g", v); }

}  // namespace

extern "C" {

int rdgpu_traj_open(const char* path, int32_t format, rdgpu_traj_handle* out)
{
    if (!out) return out_fail("rdgpu_traj_open: null output handle");
    *out = nullptr;
    if (!path || !*path) return out_fail("rdgpu_traj_open: empty path");
    if (format != RDGPU_TRAJ_XML && format != RDGPU_TRAJ_PDB)
        return out_fail("rdgpu_traj_open: format must be RDGPU_TRAJ_XML or RDGPU_TRAJ_PDB");
    FILE* f = std::fopen(path, "w");
    if (!f) return out_fail(std::string("cannot open ") + path + " for writing");
    if (format == RDGPU_TRAJ_XML && std::fputs("<traj>\n", f) < 0) {
        std::fclose(f);
        return out_fail(std::string("cannot write ") + path);
    }
    auto* t = new rdgpu_traj();
    t->f = f;
    t->format = format;
    t->path = path;
    *out = t;
    return RDGPU_OK;
}

int rdgpu_traj_write(rdgpu_traj_handle t, int64_t step, int64_t n, const double* xyz, const int32_t* types,
                     const int32_t* ids)
{
    if (!t || !t->f) return out_fail("rdgpu_traj_write: closed or null handle");
    if (n < 0 || (n > 0 && (!xyz || !types))) return out_fail("rdgpu_traj_write: n >= 0 with xyz and types needed");
    FILE* f = t->f;
    bool ok = true;
    if (t->format == RDGPU_TRAJ_XML) {
        // one frame in the coordinate-input format (CoordReader.cpp:27-40)
        ok = std::fprintf(f, "<tplgy_coords version=\"1.1\" stepId=\"%lld\">\n", (long long)step) > 0;
        for (int64_t a = 0; ok && a < n; ++a) {
            const long long id = ids ? (long long)ids[a] : (long long)(a + 1);
            std::fprintf(f, "<p id=\"%lld\" type=\"%d\" c=\"", id, (int)types[a]);
            put_coord(f, xyz[3 * a]);
            std::fputc(',', f);
            put_coord(f, xyz[3 * a + 1]);
            std::fputc(',', f);
            put_coord(f, xyz[3 * a + 2]);
            ok = std::fputs("\"/>\n", f) >= 0;
        }
        ok = ok && std::fputs("</tplgy_coords>\n", f) >= 0;
    } else {
        // PDB records in fixed columns: serial, type as name and residue,
        // x y z in 8.3, occupancy and B-factor placeholders
        ok = std::fprintf(f, "MODEL     %lld\n", (long long)step) > 0;
        for (int64_t a = 0; ok && a < n; ++a)
            ok = std::fprintf(f, "ATOM  %5lld   %i    %i     1    %8.3f%8.3f%8.3f 15.00  0.00\n", (long long)(a + 1),
                              (int)types[a], (int)types[a], xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2]) > 0;
        ok = ok && std::fputs("ENDMDL\n", f) >= 0;
    }
    if (!ok || std::ferror(f)) return out_fail("cannot write " + t->path);
    return RDGPU_OK;
}

int rdgpu_traj_close(rdgpu_traj_handle t)
{
    if (!t) return out_fail("rdgpu_traj_close: null handle");
    bool ok = true;
    if (t->f) {
        if (t->format == RDGPU_TRAJ_XML) ok = std::fputs("</traj>\n", t->f) >= 0;
        ok = (std::fclose(t->f) == 0) && ok;
    }
    const std::string path = t->path;
    delete t;
    return ok ? RDGPU_OK : out_fail("cannot finish " + path);
}

int rdgpu_write_rdf_csv(const char* path, int32_t n_types, const char* const* names, int32_t nbins, double rmax,
                        const double* g)
{
    if (!path || !*path) return out_fail("rdgpu_write_rdf_csv: empty path");
    if (n_types < 1 || nbins < 1 || !(rmax > 0.0) || !names || !g)
        return out_fail("rdgpu_write_rdf_csv: n_types >= 1, nbins >= 1, rmax > 0, names and g needed");
    for (int32_t a = 0; a < n_types; ++a)
        if (!names[a]) return out_fail("rdgpu_write_rdf_csv: null type name");
    FILE* f = std::fopen(path, "w");
    if (!f) return out_fail(std::string("cannot open ") + path + " for writing");
    bool ok = std::fputc('d', f) != EOF;
    for (int32_t a = 0; a < n_types; ++a)
        for (int32_t b = 0; b < n_types; ++b) ok = ok && std::fprintf(f, ",\tRDF(%s,%s)", names[a], names[b]) > 0;
    ok = ok && std::fputc('\n', f) != EOF;
    for (int32_t k = 0; ok && k < nbins; ++k) {
        ok = std::fprintf(f, "%8.5f", (double)k * rmax / (double)nbins) > 0;
        for (int32_t a = 0; a < n_types; ++a)
            for (int32_t b = 0; b < n_types; ++b)
                ok = ok && std::fprintf(f, ", %8.3f", g[((int64_t)a * n_types + b) * nbins + k]) > 0;
        ok = ok && std::fputc('\n', f) != EOF;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RDGPU_OK : out_fail(std::string("cannot write ") + path);
}

const char* rdgpu_output_error(void) { return g_out_err.c_str(); }

}  // extern "C"
