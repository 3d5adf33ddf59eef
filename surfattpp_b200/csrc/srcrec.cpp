// Observation table and event builder (host code; reference src/src_rec.cpp).
//   sa_srcrec_load   SrcRec::load + get_periods + get_events (:20-228, :232-264):
//                    CSV columns tt, staname, stla, stlo, evtname, evla, evlo,
//                    period [, weight, dist, vel]; one event per (sorted unique
//                    evtname, period index) with its observation rows, in the
//                    order of the reference's events map (key "{evt}_{iper}").
//   sa_srcrec_write  SrcRec::write (:407-457): observed or forward times.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "surfatt_gpu.h"

namespace {
constexpr double PI_S = 3.14159265358979323846264338327950288;
constexpr double DEG2RAD_S = PI_S / 180.0;
constexpr double R_EARTH_S = 6371.0;

// include/utils.h:287-299
double gps2dist(double lat0, double lon0, double lat1, double lon1) {
    const double dlat = (lat0 - lat1) * DEG2RAD_S;
    const double dlon = (lon1 - lon0) * DEG2RAD_S;
    const double a = std::sin(dlat * 0.5) * std::sin(dlat * 0.5) +
                     std::sin(dlon * 0.5) * std::sin(dlon * 0.5) * std::cos(lat0 * DEG2RAD_S) *
                         std::cos(lat1 * DEG2RAD_S);
    const double rad = 2.0 * std::atan2(std::sqrt(a), std::sqrt(1.0 - a));
    return R_EARTH_S * rad;
}

std::vector<std::string> split_csv(const std::string& line) {
    std::vector<std::string> out;
    std::string cur;
    bool q = false;
    for (size_t i = 0; i < line.size(); i++) {
        const char ch = line[i];
        if (q) {
            if (ch == '"' && i + 1 < line.size() && line[i + 1] == '"') {
                cur += '"';
                i++;
            } else if (ch == '"') {
                q = false;
            } else {
                cur += ch;
            }
        } else if (ch == '"') {
            q = true;
        } else if (ch == ',') {
            out.push_back(cur);
            cur.clear();
        } else if (ch != '\r') {
            cur += ch;
        }
    }
    out.push_back(cur);
    return out;
}

bool to_double(const std::string& s, double* v) {
    const char* b = s.c_str();
    char* e = nullptr;
    *v = std::strtod(b, &e);
    while (e && *e == ' ') e++;
    return e != b && e && *e == '\0';
}

std::string fixed(double v, int prec) {   // include/utils.h:664-674 (std::fixed)
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*f", prec, v);
    return buf;
}
}  // namespace

struct sa_srcrec {
    int n_obs = 0;
    std::vector<double> stla, stlo, evla, evlo, dist, period, tt, vel, weight;
    std::vector<std::string> staname, evtname;
    std::vector<double> periods, meanvel;
    std::vector<int> n_obs_per;
    // events in map-key order
    std::vector<std::string> ev_name;
    std::vector<double> ev_lo, ev_la;
    std::vector<int> ev_iper, rec_ptr, rec_idx;
    std::string err;
};

extern "C" int sa_srcrec_load(const char* path, sa_srcrec** out) {
    if (!path || !out) return SA_ERR_ARG;
    *out = nullptr;
    std::ifstream f(path);
    if (!f) return SA_ERR_ARG;
    sa_srcrec* S = new sa_srcrec();
    std::string line;
    if (!std::getline(f, line)) {
        delete S;
        return SA_ERR_ARG;
    }
    const auto hdr = split_csv(line);
    auto col = [&](const char* name) {
        for (size_t i = 0; i < hdr.size(); i++)
            if (hdr[i] == name) return (int)i;
        return -1;
    };
    const int c_stla = col("stla"), c_stlo = col("stlo"), c_evla = col("evla"),
              c_evlo = col("evlo"), c_per = col("period"), c_tt = col("tt"),
              c_evt = col("evtname"), c_sta = col("staname"), c_w = col("weight"),
              c_d = col("dist"), c_v = col("vel");
    if (c_stla < 0 || c_stlo < 0 || c_evla < 0 || c_evlo < 0 || c_per < 0 || c_tt < 0 ||
        c_evt < 0 || c_sta < 0) {
        delete S;
        return SA_ERR_ARG;
    }
    std::vector<double> dcol, vcol, wcol;
    while (std::getline(f, line)) {
        if (line.empty() || line == "\r") continue;
        const auto v = split_csv(line);
        if ((int)v.size() < (int)hdr.size()) {
            delete S;
            return SA_ERR_ARG;
        }
        double x[6];
        const int cs[6] = {c_stla, c_stlo, c_evla, c_evlo, c_per, c_tt};
        for (int k = 0; k < 6; k++)
            if (!to_double(v[cs[k]], &x[k])) {
                delete S;
                return SA_ERR_ARG;
            }
        S->stla.push_back(x[0]);
        S->stlo.push_back(x[1]);
        S->evla.push_back(x[2]);
        S->evlo.push_back(x[3]);
        S->period.push_back(x[4]);
        S->tt.push_back(x[5]);
        S->evtname.push_back(v[c_evt]);
        S->staname.push_back(v[c_sta]);
        double y;
        if (c_w >= 0) wcol.push_back(to_double(v[c_w], &y) ? y : 1.0);
        if (c_d >= 0) dcol.push_back(to_double(v[c_d], &y) ? y : 0.0);
        if (c_v >= 0) vcol.push_back(to_double(v[c_v], &y) ? y : 0.0);
    }
    const int n = (int)S->tt.size();
    S->n_obs = n;
    // optional columns (:56-80)
    S->weight = c_w >= 0 ? wcol : std::vector<double>(n, 1.0);
    if (c_d >= 0) S->dist = dcol;
    else {
        S->dist.resize(n);
        for (int i = 0; i < n; i++) S->dist[i] = gps2dist(S->stla[i], S->stlo[i], S->evla[i], S->evlo[i]);
    }
    if (c_v >= 0) S->vel = vcol;
    else {
        S->vel.resize(n);
        for (int i = 0; i < n; i++) S->vel[i] = (S->tt[i] > 0) ? (S->dist[i] / S->tt[i]) : 0.0;
    }
    // get_periods (:232-257)
    std::vector<double> pv = S->period;
    std::sort(pv.begin(), pv.end());
    pv.erase(std::unique(pv.begin(), pv.end()), pv.end());
    S->periods = pv;
    for (double per : pv) {
        int cnt = 0;
        double sv = 0.0;
        for (int j = 0; j < n; j++)
            if (std::abs(S->period[j] - per) < 1e-6) {
                cnt++;
                sv += S->vel[j];
            }
        S->n_obs_per.push_back(cnt);
        S->meanvel.push_back(sv / cnt);
    }
    // get_events (:142-178): map key "{evt}_{iper}", observation rows in order
    std::vector<std::string> keys = S->evtname;
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    struct Ev {
        double lo, la;
        int iper;
        std::vector<int> rows;
    };
    std::map<std::string, Ev> evs;
    for (const auto& src : keys)
        for (int ip = 0; ip < (int)pv.size(); ip++) {
            Ev e{0.0, 0.0, ip, {}};
            for (int i = 0; i < n; i++)
                if (S->evtname[i] == src && std::abs(pv[ip] - S->period[i]) < 1e-6) {
                    e.rows.push_back(i);
                    e.la = S->evla[i];
                    e.lo = S->evlo[i];
                }
            if (!e.rows.empty()) evs[src + "_" + std::to_string(ip)] = e;
        }
    S->rec_ptr.push_back(0);
    for (auto& [k, e] : evs) {
        S->ev_name.push_back(k);
        S->ev_lo.push_back(e.lo);
        S->ev_la.push_back(e.la);
        S->ev_iper.push_back(e.iper);
        S->rec_idx.insert(S->rec_idx.end(), e.rows.begin(), e.rows.end());
        S->rec_ptr.push_back((int)S->rec_idx.size());
    }
    *out = S;
    return SA_OK;
}

extern "C" void sa_srcrec_destroy(sa_srcrec* S) { delete S; }

extern "C" int sa_srcrec_sizes(const sa_srcrec* S, int* n_obs, int* nperiod, int* n_events) {
    if (!S) return SA_ERR_ARG;
    if (n_obs) *n_obs = S->n_obs;
    if (nperiod) *nperiod = (int)S->periods.size();
    if (n_events) *n_events = (int)S->ev_name.size();
    return SA_OK;
}

extern "C" int sa_srcrec_periods(const sa_srcrec* S, double* periods, double* meanvel,
                                 int* n_obs_per_period) {
    if (!S) return SA_ERR_ARG;
    for (size_t i = 0; i < S->periods.size(); i++) {
        if (periods) periods[i] = S->periods[i];
        if (meanvel) meanvel[i] = S->meanvel[i];
        if (n_obs_per_period) n_obs_per_period[i] = S->n_obs_per[i];
    }
    return SA_OK;
}

extern "C" int sa_srcrec_observations(const sa_srcrec* S, double* stlo, double* stla, double* tt,
                                      double* weight, double* dist, double* vel, double* period) {
    if (!S) return SA_ERR_ARG;
    const size_t b = S->n_obs * sizeof(double);
    if (stlo) std::memcpy(stlo, S->stlo.data(), b);
    if (stla) std::memcpy(stla, S->stla.data(), b);
    if (tt) std::memcpy(tt, S->tt.data(), b);
    if (weight) std::memcpy(weight, S->weight.data(), b);
    if (dist) std::memcpy(dist, S->dist.data(), b);
    if (vel) std::memcpy(vel, S->vel.data(), b);
    if (period) std::memcpy(period, S->period.data(), b);
    return SA_OK;
}

extern "C" int sa_srcrec_events(const sa_srcrec* S, double* evlo, double* evla, int* iper,
                                int* rec_ptr, int* rec_idx) {
    if (!S) return SA_ERR_ARG;
    const size_t ne = S->ev_name.size();
    for (size_t e = 0; e < ne; e++) {
        if (evlo) evlo[e] = S->ev_lo[e];
        if (evla) evla[e] = S->ev_la[e];
        if (iper) iper[e] = S->ev_iper[e];
    }
    if (rec_ptr) std::memcpy(rec_ptr, S->rec_ptr.data(), (ne + 1) * sizeof(int));
    if (rec_idx) std::memcpy(rec_idx, S->rec_idx.data(), S->rec_idx.size() * sizeof(int));
    return SA_OK;
}

extern "C" const char* sa_srcrec_event_name(const sa_srcrec* S, int e) {
    if (!S || e < 0 || e >= (int)S->ev_name.size()) return nullptr;
    return S->ev_name[e].c_str();
}

extern "C" int sa_srcrec_write(const sa_srcrec* S, const char* path, const double* tt_fwd) {
    if (!S || !path) return SA_ERR_ARG;
    if (S->n_obs == 0) return SA_ERR_ARG;   // :409-411
    std::ofstream f(path);
    if (!f) return SA_ERR_ARG;
    f << "tt,staname,stla,stlo,evtname,evla,evlo,period,weight,dist,vel\n";
    for (int i = 0; i < S->n_obs; i++) {
        const double t = tt_fwd ? tt_fwd[i] : S->tt[i];
        const double v = tt_fwd ? S->dist[i] / tt_fwd[i] : S->vel[i];   // :366-370
        f << fixed(t, 6) << ',' << S->staname[i] << ',' << fixed(S->stla[i], 4) << ','
          << fixed(S->stlo[i], 4) << ',' << S->evtname[i] << ',' << fixed(S->evla[i], 4) << ','
          << fixed(S->evlo[i], 4) << ',' << fixed(S->period[i], 2) << ','
          << fixed(S->weight[i], 4) << ',' << fixed(S->dist[i], 3) << ',' << fixed(v, 6) << '\n';
    }
    return f.good() ? SA_OK : SA_ERR_ARG;
}
