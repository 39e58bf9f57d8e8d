/* Test infrastructure only (the checker, never the product path).
 *
 * The reference's CDM driver (reg/cdm.hpp:19-34, 373-474) restated in plain C for
 * a list of modalities.  Included after oracle_core.h and oracle_field.h with the same
 * SFX/PIX/R and FSFX macros.
 */
#define DCAT_(a, b) a##b
#define DCAT(a, b) DCAT_(a, b)
#define DN(name) DCAT(name, SFX)
#define DF(name) DCAT(name, FSFX)

/* cdm_improved (reg/cdm.hpp:19-34): once more than 5 costs are held, fit
 * cost = a*iter + b (statistics.hpp:694-713 with int x and float y, cross
 * products in float); a rising trend means "not improved".  Beyond 7 costs the
 * oldest is dropped.  cost/len are updated in place. */
static int DN(cdm_improved)(R* cost, int* len)
{
    int n = *len;
    if (n > 5) {
        long long sx = 0, sxx = 0;
        double sy = cost[0], syy = 0, sxy = (double)(R)(0 * cost[0]);
        for (int i = 0; i < n; ++i) {
            sx += i;
            sxx += (long long)i * i;
        }
        for (int i = 1; i < n; ++i) {
            sy += cost[i];
            sxy += (double)((R)i * cost[i]);
        }
        for (int i = 0; i < n; ++i) {
            double t = cost[i];
            syy += t * t;
        }
        double mx = (double)sx / n, my = sy / n;
        double xv = (double)sxx / n - mx * mx, yv = syy / n - my * my;
        R a = 0;
        if (!(xv == 0 || yv == 0)) {
            double cov = sxy / n - mx * my;
            a = (R)(cov / xv);
        }
        if (a > 0)
            return 0;
        if (n > 7) {
            for (int i = 1; i < n; ++i)
                cost[i - 1] = cost[i];
            *len = n - 1;
        }
    }
    return 1;
}

typedef struct {
    float resolution, speed, smoothing;
    unsigned int min_dimension;
    int gradient_type; /* 'r' or 'd' */
} DN(orc_cdm_param_t);

/* cdm(It, Is, best_d, terminated, param) (reg/cdm.hpp:373-474) over nmod modality
 * pairs It[i] / Is[i] of one shape.  Each iteration composes and differentiates every
 * modality in turn (reg/cdm.hpp:419-435): the gradients are summed into new_d in
 * modality order (new_d = dd0, new_d += dd1, ...), the float costs into sum_cost, which
 * fails the call as soon as a partial sum is exactly zero, and the iteration's cost is
 * sum_cost / nmod.  Modality i uses gtypes[i] ('r' or 'd'), 'r' past the string's end.
 * best_d holds dim[0]*dim[1]*dim[2]*3 values and must start zeroed.  iters_out (may be
 * NULL) accumulates the number of iterations run over all levels.  Returns 0 where the
 * reference returns false (a zero cost sum). */
int DN(orc_cdm_multi)(const PIX* const* It, const PIX* const* Is, int nmod, const int* dim, R* best_d,
                      float resolution, float speed, float smoothing, unsigned int min_dimension, const char* gtypes,
                      int* iters_out)
{
    long long n = (long long)dim[0] * dim[1] * dim[2];
    int ntype = gtypes ? (int)strlen(gtypes) : 0;
    int mn = dim[0];
    if (dim[1] < mn) mn = dim[1];
    if (dim[2] < mn) mn = dim[2];
    if ((unsigned int)mn > min_dimension) {
        int rd[3] = {(dim[0] + 1) / 2, (dim[1] + 1) / 2, (dim[2] + 1) / 2};
        long long rn = (long long)rd[0] * rd[1] * rd[2];
        PIX** rIt = (PIX**)malloc(sizeof(PIX*) * nmod);
        PIX** rIs = (PIX**)malloc(sizeof(PIX*) * nmod);
        for (int i = 0; i < nmod; ++i) {
            rIt[i] = (PIX*)malloc(sizeof(PIX) * rn);
            rIs[i] = (PIX*)malloc(sizeof(PIX) * rn);
            DN(orc_downsample)(It[i], dim, rIt[i]);
            DN(orc_downsample)(Is[i], dim, rIs[i]);
        }
        R* rd_field = (R*)calloc(3 * rn, sizeof(R));
        int ok = DN(orc_cdm_multi)((const PIX* const*)rIt, (const PIX* const*)rIs, nmod, rd, rd_field,
                                   resolution / 2.0f, speed, smoothing, min_dimension, gtypes, iters_out);
        for (int i = 0; i < nmod; ++i) {
            free(rIt[i]);
            free(rIs[i]);
        }
        free(rIt);
        free(rIs);
        if (!ok) {
            free(rd_field);
            return 0;
        }
        DF(orc_upsample_field_x2)(rd_field, rd, best_d, dim);
        free(rd_field);
        if (resolution > 1.0f)
            return 1;
    }
    R theta = 0;
    R cost[8];
    int ncost = 0;
    R best_cost = (R)3.402823466e+38f;
    R* cur_d = (R*)malloc(sizeof(R) * 3 * n);
    R* new_d = (R*)malloc(sizeof(R) * 3 * n);
    R* dd = nmod > 1 ? (R*)malloc(sizeof(R) * 3 * n) : NULL;
    PIX* Js = (PIX*)malloc(sizeof(PIX) * n);
    memcpy(cur_d, best_d, sizeof(R) * 3 * n);
    R cur_smoothing = (R)0.8f;
    int ok = 1;
    for (unsigned int index = 0; index < 200 && ok; ++index) {
        R sum_cost = 0;
        for (int i = 0; i < nmod; ++i) {
            DN(orc_compose)(Is[i], dim, cur_d, Js);
            R* out = i ? dd : new_d;
            sum_cost += DN(orc_cdm_gradient)(Js, It[i], dim, out, i < ntype ? gtypes[i] : 'r');
            if (sum_cost == 0) {
                ok = 0;
                break;
            }
            if (i)
                for (long long k = 0; k < 3 * n; ++k)
                    new_d[k] += dd[k];
        }
        if (!ok)
            break;
        if (iters_out)
            ++*iters_out;
        cost[ncost++] = sum_cost / (R)nmod;
        if (cost[ncost - 1] < best_cost) {
            best_cost = cost[ncost - 1];
            if (index)
                memcpy(best_d, cur_d, sizeof(R) * 3 * n);
        }
        if (!DN(cdm_improved)(cost, &ncost)) {
            if (cur_smoothing <= (R)smoothing)
                break;
            memcpy(cur_d, best_d, sizeof(R) * 3 * n);
            cur_smoothing *= (R)0.5f;
            ncost = 0;
        }
        DF(orc_cdm_poisson)(new_d, dim, 12);
        if (theta == 0)
            theta = DF(orc_cdm_max_len)(new_d, dim);
        if (theta == 0)
            break;
        DF(orc_field_scale)(new_d, dim, (R)speed / theta);
        DF(orc_accumulate)(cur_d, new_d, dim);
        DF(orc_cdm_smooth)(new_d, cur_d, dim, cur_smoothing);
    }
    free(cur_d);
    free(new_d);
    free(dd);
    free(Js);
    return ok;
}

/* The one-modality call (cdm_common with single-image lists). */
int DN(orc_cdm_level)(const PIX* It, const PIX* Is, const int* dim, R* best_d, float resolution, float speed,
                      float smoothing, unsigned int min_dimension, int gradient_type, int* iters_out)
{
    char gt[2] = {(char)gradient_type, 0};
    return DN(orc_cdm_multi)(&It, &Is, 1, dim, best_d, resolution, speed, smoothing, min_dimension, gt, iters_out);
}

#undef DN
#undef DF
#undef DCAT
#undef DCAT_
