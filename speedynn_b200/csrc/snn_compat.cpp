// snn_compat.cpp -- the drop-in layer: speedynn's SWIG-level C API
// (speedynn/lib/nearest_neighbors_feature_selection.h:59-80) implemented on
// top of the handle API, plus the host-side loss utility get_loss_all.
//
// Behaviour kept from the reference: CV mode over one training matrix, the
// results of the last run live in library state read by the get_* functions,
// the return value is the final number of features.  Behaviour changed on
// purpose: no exit()/printf on errors (negative status + snn_last_error()),
// and the n > 15000 "large scale" exit (nearest_neighbors_feature_selection.c:84-87)
// does not exist.  Loss lists and the classification model are passed to
// snn_set_model; an unknown model type or loss id is rejected with
// SNN_ERR_UNSUPPORTED instead of running undefined code.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/speedynn_b200.h"

namespace {

struct LastRun {
    std::vector<int> mask, order;
    std::vector<float> errors;  // [num_losses][p]
    int best_k = 0;
};

std::mutex g_mu;
LastRun g_last;

int train_common(int backward, float *X, int n, int d, float *y, int ny, int *kvals, int nk, int num_features, int kfold,
                 int *loss_functions, int nl, int auto_feature, int model_type)
{
    if (!X || !y || !kvals || n <= 0 || d <= 0 || ny != n || nk <= 0) return SNN_ERR_ARG;
    if (model_type != 0 && model_type != 1) return SNN_ERR_UNSUPPORTED;
    if (nl < 0 || (nl > 0 && !loss_functions)) return SNN_ERR_ARG;
    static const int kRmseOnly[1] = {SNN_LOSS_RMSE};
    const int *ids = nl > 0 ? loss_functions : kRmseOnly;
    const int n_ids = nl > 0 ? nl : 1;
    for (int l = 0; l < n_ids; ++l)
        if (ids[l] < 0 || ids[l] > 8) return SNN_ERR_UNSUPPORTED;
    snn_desc desc;
    memset(&desc, 0, sizeof desc);
    desc.n_train = n;
    desc.n_val = 0;
    desc.p = d;
    desc.k_vals = kvals;
    desc.num_k_vals = nk;
    desc.backward = backward;
    desc.num_features = num_features;
    desc.k_fold = kfold;
    desc.auto_feature = auto_feature;
    desc.device = 0;
    if (const char *dev = getenv("SNN_DEVICE")) desc.device = atoi(dev);
    snn_handle *h = nullptr;
    int rc = snn_create(&desc, &h);
    if (rc) return rc;
    rc = snn_set_model(h, ids, n_ids, model_type);
    if (!rc) rc = snn_load(h, X, y, nullptr, nullptr);
    if (!rc) rc = snn_run(h);
    LastRun r;
    r.mask.assign(d, 0);
    r.order.assign(d, 0);
    r.errors.assign((size_t)n_ids * d, 0.0f);
    int num_final = 0;
    if (!rc) rc = snn_get_results(h, r.order.data(), r.mask.data(), nullptr, nullptr, nullptr, &r.best_k, &num_final);
    if (!rc) rc = snn_get_errors_all(h, r.errors.data(), (int)r.errors.size());
    snn_destroy(h);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    g_last = std::move(r);
    return num_final;
}

template <typename T>
void copy_out(const std::vector<T> &src, T *dst, int n)
{
    if (!dst || n <= 0) return;
    std::lock_guard<std::mutex> lk(g_mu);
    const int m = std::min<int>(n, (int)src.size());
    for (int i = 0; i < m; ++i) dst[i] = src[i];
}

// ---- losses, speedynn/lib/loss_functions.c (same float/double op order) ----

float rmse_loss(const float *labels, const float *preds, int num)
{
    float sum = 0.0f;
    for (int i = 0; i < num; i++) {
        float tmp = labels[i] - preds[i];
        sum += tmp * tmp;
    }
    sum /= (float)num;
    return (float)sqrt((double)sum);
}

float rmse_norm_loss(const float *labels, const float *preds, int num)
{
    float sum = 0.0f;
    for (int i = num; i--;) {
        float t = labels[i];
        float tmp = (float)((double)(t - preds[i]) / (1.0 + (double)t));
        sum += tmp * tmp;
    }
    sum /= (float)num;
    return (float)sqrt((double)sum);
}

float median_of(std::vector<float> v)
{
    std::sort(v.begin(), v.end());
    return v[v.size() / 2];
}

float mad_generic(const float *labels, const float *preds, int num, bool norm)
{
    std::vector<float> e(num);
    for (int i = 0; i < num; i++) {
        float t = labels[i];
        e[i] = norm ? (float)((double)(t - preds[i]) / (1.0 + (double)t)) : (t - preds[i]);
    }
    float m1 = median_of(e);
    for (int i = 0; i < num; i++) e[i] = (float)fabs((double)(e[i] - m1));
    return median_of(e);
}

float zero_one_loss(const float *labels, const float *preds, int num)
{
    // loss_functions.c:119 passes a float to int abs(): the difference is
    // truncated to int, so only |t - p| >= 1 counts as a miss.
    float sum = 0.0f;
    for (int i = 0; i < num; i++) {
        const int tr = (int)(labels[i] - preds[i]);
        sum += (abs(tr) < 10E-8) ? 0.0f : 1.0f;
    }
    sum /= (float)num;
    return sum;
}

float std_loss(const float *labels, const float *preds, int num)
{
    float mean = 0.0f;
    for (int i = 0; i < num; i++) mean += (labels[i] - preds[i]);
    mean /= (float)num;
    float sum = 0.0f;
    for (int i = 0; i < num; i++) {
        // loss_functions.c:141 assigns instead of accumulating
        float a = (labels[i] - preds[i]) - mean;
        sum = a * a;
    }
    sum /= (float)(num - 1);
    return (float)sqrt((double)sum);
}

}  // namespace

extern "C" {

SNN_API int train_forward_selection(float *Xtrain, int nXtrain, int dXtrain, float *Ytrain, int nYtrain, int *kvals,
                                    int num_kvals, int num_features, int kfold, int *loss_functions,
                                    int num_loss_functions, int auto_feature, int model_type)
{
    return train_common(0, Xtrain, nXtrain, dXtrain, Ytrain, nYtrain, kvals, num_kvals, num_features, kfold,
                        loss_functions, num_loss_functions, auto_feature, model_type);
}

SNN_API int train_backward_selection(float *Xtrain, int nXtrain, int dXtrain, float *Ytrain, int nYtrain, int *kvals,
                                     int num_kvals, int num_features, int kfold, int *loss_functions,
                                     int num_loss_functions, int auto_feature, int model_type)
{
    return train_common(1, Xtrain, nXtrain, dXtrain, Ytrain, nYtrain, kvals, num_kvals, num_features, kfold,
                        loss_functions, num_loss_functions, auto_feature, model_type);
}

SNN_API void get_selected_dimensions(int *out, int n) { copy_out(g_last.mask, out, n); }
SNN_API void get_selected_ordering(int *out, int n) { copy_out(g_last.order, out, n); }
SNN_API void get_selected_errors(float *out, int n) { copy_out(g_last.errors, out, n); }

SNN_API int get_final_optimal_model_k(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_last.best_k;
}

SNN_API float get_loss_all(float *labels, int num_labels, float *predictions, int num_predictions, int loss_function)
{
    if (!labels || !predictions || num_labels <= 0 || num_labels != num_predictions) return NAN;
    const int n = num_labels;
    switch (loss_function) {
    case 0: return rmse_loss(labels, predictions, n);
    case 1: return rmse_norm_loss(labels, predictions, n);
    case 2: return mad_generic(labels, predictions, n, false);
    case 3: return mad_generic(labels, predictions, n, true);
    case 4: return zero_one_loss(labels, predictions, n);
    case 5: return std_loss(labels, predictions, n);
    case 6: {
        const float a = rmse_norm_loss(labels, predictions, n);
        const float b = mad_generic(labels, predictions, n, true);
        const float c = std_loss(labels, predictions, n);
        return (float)((double)a / 0.19 + (double)b / 0.041 + (double)c / 0.16);
    }
    case 7: {
        const float a = rmse_norm_loss(labels, predictions, n);
        const float b = mad_generic(labels, predictions, n, true);
        return (float)((double)a / 0.019 + (double)b / 0.009);
    }
    case 8: return rmse_loss(labels, predictions, n) + std_loss(labels, predictions, n);
    default: return NAN;
    }
}

}  // extern "C"
