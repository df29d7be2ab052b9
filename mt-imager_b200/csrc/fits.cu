// FITS cube writer (include/mtb_fits.h), host code only.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <algorithm>
#include <vector>

#include "mtb_fits.h"

struct mtb_fits {
    FILE *f = nullptr;
    size_t data_offset = 0;
    size_t channel_bytes = 0;
    int nchan = 0;
};

namespace {

const size_t kBlock = 2880;

std::string card(const char *key, const std::string &value, const char *comment = nullptr) {
    char buf[96];
    if (comment)
        std::snprintf(buf, sizeof(buf), "%-8.8s= %20s / %s", key, value.c_str(), comment);
    else
        std::snprintf(buf, sizeof(buf), "%-8.8s= %20s", key, value.c_str());
    std::string s(buf);
    s.resize(80, ' ');
    return s;
}
std::string num(double v) {
    char b[40];
    std::snprintf(b, sizeof(b), "%.15G", v);
    std::string s(b);
    if (s.find_first_of(".EN") == std::string::npos) s += ".";
    return s;
}
std::string integer(long long v) { return std::to_string(v); }
std::string str(const std::string &v) {
    std::string q;
    for (char c : v) {
        q += c;
        if (c == '\'') q += '\'';
    }
    std::string s = "'" + q;
    while (s.size() < 9) s += ' ';    // fixed-format strings are at least 8 characters
    return s + "'";
}
std::string iso_date(double mjd) {
    // MJD (UTC) to YYYY-MM-DDThh:mm:ss.sss
    const double days = mjd - 40587.0;   // MJD of 1970-01-01
    const double secs = days * 86400.0;
    std::time_t t = (std::time_t)std::floor(secs);
    std::tm tm;
    gmtime_r(&t, &tm);
    char b[40];
    std::snprintf(b, sizeof(b), "%04d-%02d-%02dT%02d:%02d:%06.3f", tm.tm_year + 1900, tm.tm_mon + 1, tm.tm_mday,
                  tm.tm_hour, tm.tm_min, tm.tm_sec + (secs - std::floor(secs)));
    return b;
}

}  // namespace

extern "C" int mtb_fits_create(const char *path, const mtb_fits_header *h, mtb_fits **out) {
    if (!path || !h || !out) return MTB_ERR_NULL;
    *out = nullptr;
    if (h->nx < 1 || h->ny < 1 || h->nstokes < 1 || h->nchan < 1) return MTB_ERR_BAD_SHAPE;
    if (!h->freqs_hz || !h->stokes) return MTB_ERR_NULL;
    const double rad2deg = 180.0 / M_PI;
    std::vector<std::string> cards;
    cards.push_back(card("SIMPLE", "T", "conforms to FITS"));
    cards.push_back(card("BITPIX", integer(-32), "Floating point (32 bit)"));
    cards.push_back(card("NAXIS", integer(4)));
    cards.push_back(card("NAXIS1", integer(h->nx)));
    cards.push_back(card("NAXIS2", integer(h->ny)));
    cards.push_back(card("NAXIS3", integer(h->nstokes)));
    cards.push_back(card("NAXIS4", integer(h->nchan)));
    cards.push_back(card("EXTEND", "T"));
    cards.push_back(card("BSCALE", num(1.0), "PHYSICAL = PIXEL*BSCALE + BZERO"));
    cards.push_back(card("BZERO", num(0.0)));
    cards.push_back(card("BUNIT", str("JY/BEAM"), "Brightness (pixel) unit"));
    cards.push_back(card("CTYPE1", str("RA---SIN")));
    cards.push_back(card("CRVAL1", num(h->ra_deg)));
    cards.push_back(card("CDELT1", num(-h->l_increment * rad2deg)));
    cards.push_back(card("CRPIX1", num((double)(h->nx / 2) + 1.0)));
    cards.push_back(card("CUNIT1", str("deg")));
    cards.push_back(card("CTYPE2", str("DEC--SIN")));
    cards.push_back(card("CRVAL2", num(h->dec_deg)));
    cards.push_back(card("CDELT2", num(h->m_increment * rad2deg)));
    cards.push_back(card("CRPIX2", num((double)(h->ny / 2) + 1.0)));
    cards.push_back(card("CUNIT2", str("deg")));
    cards.push_back(card("CTYPE3", str("STOKES")));
    cards.push_back(card("CRVAL3", num((double)h->stokes[0])));
    cards.push_back(card("CDELT3", num(h->nstokes > 1 ? (double)(h->stokes[1] - h->stokes[0]) : 1.0)));
    cards.push_back(card("CRPIX3", num(1.0)));
    cards.push_back(card("CUNIT3", str("")));
    const double df = h->nchan > 1 ? (h->freqs_hz[h->nchan - 1] - h->freqs_hz[0]) / (h->nchan - 1) : 1.0;
    cards.push_back(card("CTYPE4", str("FREQ")));
    cards.push_back(card("CRVAL4", num(h->freqs_hz[0])));
    cards.push_back(card("CDELT4", num(df)));
    cards.push_back(card("CRPIX4", num(1.0)));
    cards.push_back(card("CUNIT4", str("Hz")));
    cards.push_back(card("SPECSYS", str("LSRK")));
    cards.push_back(card("RADESYS", str("FK5")));
    cards.push_back(card("EQUINOX", num(2000.0)));
    cards.push_back(card("LONPOLE", num(180.0)));
    cards.push_back(card("LATPOLE", num(h->dec_deg)));
    if (h->telescope) cards.push_back(card("TELESCOP", str(h->telescope)));
    if (h->observer) cards.push_back(card("OBSERVER", str(h->observer)));
    // ObsInfo's pointing centre is the phase centre (ImageManager.cpp:100)
    cards.push_back(card("OBSRA", num(h->ra_deg)));
    cards.push_back(card("OBSDEC", num(h->dec_deg)));
    if (h->obs_mjd > 0) cards.push_back(card("DATE-OBS", str(iso_date(h->obs_mjd))));
    const double now_mjd = (double)std::time(nullptr) / 86400.0 + 40587.0;
    cards.push_back(card("DATE", str(iso_date(now_mjd)), "Date FITS file was written"));
    cards.push_back(card("TIMESYS", str("UTC"), "Time system for HDU"));
    cards.push_back(card("ORIGIN", str("mtb: W-projection imaging on B200")));
    std::string endc = "END";
    endc.resize(80, ' ');
    cards.push_back(endc);
    std::string header;
    for (auto &c : cards) header += c;
    header.resize((header.size() + kBlock - 1) / kBlock * kBlock, ' ');

    FILE *f = std::fopen(path, "wb+");
    if (!f) return MTB_ERR_BAD_PARAM;
    std::unique_ptr<mtb_fits> m(new mtb_fits());
    m->f = f;
    m->data_offset = header.size();
    m->channel_bytes = (size_t)h->nx * h->ny * h->nstokes * 4;
    m->nchan = h->nchan;
    bool ok = std::fwrite(header.data(), 1, header.size(), f) == header.size();
    // zero-filled data area padded to whole blocks
    const size_t data = m->channel_bytes * h->nchan;
    const size_t padded = (data + kBlock - 1) / kBlock * kBlock;
    std::vector<char> zeros(1 << 20, 0);
    for (size_t done = 0; ok && done < padded; done += zeros.size())
        ok = std::fwrite(zeros.data(), 1, std::min(zeros.size(), padded - done), f) ==
             std::min(zeros.size(), padded - done);
    if (!ok) {
        std::fclose(f);
        return MTB_ERR_CAPACITY;
    }
    *out = m.release();
    return MTB_OK;
}

extern "C" int mtb_fits_write_channel(mtb_fits *m, int chan, const float *image) {
    if (!m || !image) return MTB_ERR_NULL;
    if (chan < 0 || chan >= m->nchan) return MTB_ERR_BAD_SHAPE;
    const size_t n = m->channel_bytes / 4;
    std::vector<uint32_t> be(n);
    for (size_t i = 0; i < n; i++) {
        uint32_t v;
        std::memcpy(&v, image + i, 4);
        be[i] = __builtin_bswap32(v);
    }
    if (std::fseek(m->f, (long)(m->data_offset + m->channel_bytes * chan), SEEK_SET) != 0) return MTB_ERR_CAPACITY;
    if (std::fwrite(be.data(), 4, n, m->f) != n) return MTB_ERR_CAPACITY;
    return MTB_OK;
}

extern "C" int mtb_fits_close(mtb_fits *m) {
    if (!m) return MTB_ERR_NULL;
    const int r = std::fclose(m->f) == 0 ? MTB_OK : MTB_ERR_CAPACITY;
    delete m;
    return r;
}
