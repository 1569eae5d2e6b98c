/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Compiles the reference's src/KernelSampler.cpp unmodified (textual include)
 * and exposes its phase function, sun light and tables through C entry points:
 *   miepdf / miecdf tables      src/KernelSampler.cpp:8-141
 *   MiePhase::Evaluate/RGB/Sample src/KernelSampler.cpp:214-285
 *   SunLight::Evaluate/Pdf/Sample src/KernelSampler.cpp:305-345
 */
#include "KernelSampler.cpp"

#include <cstring>

extern "C" unsigned ref_mie_table_size(void) { return miedl; }

extern "C" void ref_mie_tables(float *pdf_rgb, float *cdf_rgb) {
    for (unsigned i = 0; i < miedl; ++i) {
        pdf_rgb[3 * i + 0] = miepdf[i].x;
        pdf_rgb[3 * i + 1] = miepdf[i].y;
        pdf_rgb[3 * i + 2] = miepdf[i].z;
        cdf_rgb[3 * i + 0] = miecdf[i].x;
        cdf_rgb[3 * i + 1] = miecdf[i].y;
        cdf_rgb[3 * i + 2] = miecdf[i].z;
    }
}

static sfloat1 lane0(float v) { return sfloat1(v, 0.0f, 0.0f, 0.0f); }

extern "C" void ref_mie_eval(const float *ct, unsigned n, float *out_scalar, float *out_rgb) {
    for (unsigned i = 0; i < n; ++i) {
        sfloat1 c = lane0(ct[i]);
        sfloat1 s = KernelSampler::MiePhase::gmie.Evaluate(c);
        sfloat4 r = KernelSampler::MiePhase::gmie.EvaluateRGB(c);
        out_scalar[i] = s.get<0>();
        for (int k = 0; k < 3; ++k) out_rgb[3 * i + k] = r.v[k].get<0>();
    }
}

extern "C" void ref_mie_sample(const float *iv3, const float *u1, const float *u2, unsigned n, float *out3) {
    for (unsigned i = 0; i < n; ++i) {
        sfloat4 iv;
        for (int k = 0; k < 3; ++k) iv.v[k] = lane0(iv3[3 * i + k]);
        iv.v[3] = sfloat1::zero();
        sfloat4 d = KernelSampler::MiePhase::gmie.Sample(iv, lane0(u1[i]), lane0(u2[i]));
        for (int k = 0; k < 3; ++k) out3[3 * i + k] = d.v[k].get<0>();
    }
}

extern "C" void ref_sun_ops(const float dir[3], const float color[3], float angle,
                            const float *v3, const float *u1, const float *u2, unsigned n,
                            float *eval_rgb, float *pdf, float *sample3) {
    dfloat3 D(dir[0], dir[1], dir[2]);
    dfloat3 C(color[0], color[1], color[2]);
    /* The constructor registers the light in BaseLight::lights; unregister it. */
    KernelSampler::SunLight *sun = new KernelSampler::SunLight(&D, &C, angle);
    KernelSampler::BaseLight::lights.pop_back();
    for (unsigned i = 0; i < n; ++i) {
        sfloat4 v;
        for (int k = 0; k < 3; ++k) v.v[k] = lane0(v3[3 * i + k]);
        v.v[3] = sfloat1::zero();
        sfloat4 e = sun->Evaluate(v);
        for (int k = 0; k < 3; ++k) eval_rgb[3 * i + k] = e.v[k].get<0>();
        pdf[i] = sun->Pdf(v).get<0>();
        sfloat4 s = sun->Sample(v, lane0(u1[i]), lane0(u2[i]));
        for (int k = 0; k < 3; ++k) sample3[3 * i + k] = s.v[k].get<0>();
    }
    delete sun;
}

/* HGPhase::Evaluate / Sample (src/KernelSampler.cpp:164-204) with g1 = g. */
extern "C" void ref_hg_eval(float g, const float *ct, unsigned n, float *out) {
    KernelSampler::HGPhase hg(g);
    for (unsigned i = 0; i < n; ++i) out[i] = hg.Evaluate(lane0(ct[i])).get<0>();
}

extern "C" void ref_hg_sample(float g, const float *iv3, const float *u1, const float *u2, unsigned n, float *out3) {
    KernelSampler::HGPhase hg(g);
    for (unsigned i = 0; i < n; ++i) {
        sfloat4 iv;
        for (int k = 0; k < 3; ++k) iv.v[k] = lane0(iv3[3 * i + k]);
        iv.v[3] = sfloat1::zero();
        sfloat4 d = hg.Sample(iv, lane0(u1[i]), lane0(u2[i]));
        for (int k = 0; k < 3; ++k) out3[3 * i + k] = d.v[k].get<0>();
    }
}

/* sfloat1::atan2 (src/smmath.inl:430-445). */
extern "C" void ref_atan2(const float *y, const float *x, unsigned n, float *out) {
    for (unsigned i = 0; i < n; ++i) out[i] = sfloat1::atan2(lane0(y[i]), lane0(x[i])).get<0>();
}

/* MapEnv::Evaluate (src/KernelSampler.cpp:384-417) on a w x h RGBA map. */
extern "C" void ref_env_eval(unsigned w, unsigned h, const float *rgba, const float *rd3, unsigned n, float *out3) {
    KernelSampler::MapEnv env;
    dfloat4 *t = env.Initialize(w, h);
    std::memcpy((void *)t, rgba, (size_t)w * h * 16);
    for (unsigned i = 0; i < n; ++i) {
        sfloat4 v;
        for (int k = 0; k < 3; ++k) v.v[k] = lane0(rd3[3 * i + k]);
        v.v[3] = sfloat1::zero();
        sfloat4 e = env.Evaluate(v);
        for (int k = 0; k < 3; ++k) out3[3 * i + k] = e.v[k].get<0>();
    }
    env.Destroy();
}
