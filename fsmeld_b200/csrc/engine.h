// Host-side declarations shared by the engine and the reference-compatible
// file drivers.
#pragma once

#include <string>
#include <vector>

namespace fsm {

// A query prepared exactly as the reference prepares it (src/fsmeld.cpp:622-643,
// src/find_t_lp.cpp tables); see prepare_query.
struct HostQuery {
    int m = 0, w = 0, metric = 0, p = 0;
    double arg = 0.0;
    std::vector<double> qn, LQ, UQ, qs, pw, Dq, tlq, tuq, opw, oD, otl, otu;
    std::vector<int> ordA_l, ordB_l, ordA_u, ordB_u;
};

// raw: the query is used as given (no z-normalisation; raw mode)
int prepare_query(const double* q, int m, int metric, int w, double arg, HostQuery* hq, bool raw = false);
int macro_length(int m, long long available);
extern thread_local std::string g_last_error;

}  // namespace fsm
