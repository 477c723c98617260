/*
 * lt_fits.cpp -- map output as a FITS primary image (lt_write_fits), without cfitsio.
 *
 * The reference writes each map with cfitsio (module_writeFits_Image,
 * src/module_writeFits.cpp:113-206): a 2-D float32 primary array (BITPIX = -32, NAXIS1 =
 * nx, NAXIS2 = ny, row j of the map as image row j + 1), then the keywords BZERO = 0,
 * BSCALE = 1, a linear WCS in arcsec with the reference pixel 1 at (xmin, ymin) and
 * CDELT = (max - min)/(n - 1), ORIGIN = 'JPK-SOFT' and DATE.  The same HDU is written
 * here directly in the FITS format (NASA/IAU FITS Standard 4.0: 2880-byte blocks of
 * 80-character header cards, big-endian IEEE data, zero padding), the float keyword
 * values as cfitsio formats a float (7 significant digits).
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "../../include/lt_b200.h"

namespace {

constexpr size_t kBlock = 2880;

std::string card(const char *key, const std::string &value, const char *comment, bool quoted)
{
    char buf[81];
    std::string v = value;
    if (quoted) {
        std::string s = "'" + value;
        while (s.size() < 9) s += ' '; /* at least 8 characters inside the quotes */
        v = s + "'";
        snprintf(buf, sizeof(buf), "%-8.8s= %-20s / %s", key, v.c_str(), comment);
    } else {
        snprintf(buf, sizeof(buf), "%-8.8s= %20s / %s", key, v.c_str(), comment);
    }
    std::string c(buf);
    c.resize(80, ' ');
    return c;
}

std::string fmt_int(long v)
{
    char b[32];
    snprintf(b, sizeof(b), "%ld", v);
    return b;
}

/* a float keyword value: %.7G with a decimal point or exponent always present */
std::string fmt_float(float f)
{
    char b[40];
    snprintf(b, sizeof(b), "%.7G", (double)f);
    std::string s(b);
    if (s.find('.') == std::string::npos) {
        const size_t e = s.find('E');
        if (e == std::string::npos)
            s += ".";
        else
            s.insert(e, ".");
    }
    return s;
}

void put_be32(unsigned char *p, float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    p[0] = (unsigned char)(u >> 24);
    p[1] = (unsigned char)(u >> 16);
    p[2] = (unsigned char)(u >> 8);
    p[3] = (unsigned char)u;
}

} // namespace

extern "C" lt_status lt_write_fits(const char *path, const double *map, int32_t nx, int32_t ny,
                                   const lt_frame *frame)
{
    if (!path || !map || !frame || nx < 2 || ny < 2) return LT_ERR_INVALID_ARGUMENT;
    std::vector<std::string> cards;
    cards.push_back(card("SIMPLE", "T", "file does conform to FITS standard", false));
    cards.push_back(card("BITPIX", "-32", "number of bits per data pixel", false));
    cards.push_back(card("NAXIS", "2", "number of data axes", false));
    cards.push_back(card("NAXIS1", fmt_int(nx), "length of data axis 1", false));
    cards.push_back(card("NAXIS2", fmt_int(ny), "length of data axis 2", false));
    cards.push_back(card("EXTEND", "T", "FITS dataset may contain extensions", false));
    /* src/module_writeFits.cpp:157-195: keyword values as floats */
    const float crval1 = (float)frame->xmin, cdelt1 = (float)((frame->xmax - frame->xmin) / (nx - 1));
    const float crval2 = (float)frame->ymin, cdelt2 = (float)((frame->ymax - frame->ymin) / (ny - 1));
    cards.push_back(card("BZERO", fmt_float(0.f), "BZERO", false));
    cards.push_back(card("BSCALE", fmt_float(1.f), "BSCALE", false));
    cards.push_back(card("CRVAL1", fmt_float(crval1), "CRVAL1", false));
    cards.push_back(card("CRPIX1", fmt_float(1.f), "CRPIX1", false));
    cards.push_back(card("CDELT1", fmt_float(cdelt1), "CDELT1", false));
    cards.push_back(card("CUNIT1", "arcsec", "CUNIT1", true));
    cards.push_back(card("CTYPE1", "LINEAR", "CTYPE1", true));
    cards.push_back(card("CRVAL2", fmt_float(crval2), "CRVAL2", false));
    cards.push_back(card("CRPIX2", fmt_float(1.f), "CRPIX2", false));
    cards.push_back(card("CDELT2", fmt_float(cdelt2), "CDELT2", false));
    cards.push_back(card("CUNIT2", "arcsec", "CUNIT2", true));
    cards.push_back(card("CTYPE2", "LINEAR", "CTYPE2", true));
    cards.push_back(card("ORIGIN", "JPK-SOFT", "ORIGIN", true));
    char date[32];
    const time_t now = time(nullptr);
    struct tm t;
    gmtime_r(&now, &t);
    strftime(date, sizeof(date), "%Y-%m-%dT%H:%M:%S", &t);
    cards.push_back(card("DATE", date, "file creation date (YYYY-MM-DDThh:mm:ss UT)", true));
    std::string end = "END";
    end.resize(80, ' ');
    cards.push_back(end);
    std::string header;
    for (const std::string &c : cards) header += c;
    header.resize((header.size() + kBlock - 1) / kBlock * kBlock, ' ');
    const size_t nbytes = (size_t)nx * ny * 4;
    std::vector<unsigned char> data((nbytes + kBlock - 1) / kBlock * kBlock, 0);
    for (size_t k = 0; k < (size_t)nx * ny; k++) put_be32(&data[4 * k], (float)map[k]);
    FILE *f = fopen(path, "wb");
    if (!f) return LT_ERR_INVALID_ARGUMENT;
    const bool ok = fwrite(header.data(), 1, header.size(), f) == header.size() &&
                    fwrite(data.data(), 1, data.size(), f) == data.size();
    const bool closed = fclose(f) == 0;
    return ok && closed ? LT_OK : LT_ERR_INVALID_ARGUMENT;
}
