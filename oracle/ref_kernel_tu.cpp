/* ORACLE TEST INFRASTRUCTURE — not product code.
 *
 * Compiles the reference's src/kernel.cpp unmodified (textual include from
 * the reference tree, path supplied by -I at build time) and adds C entry
 * points for its file-local helpers so tests can pin them:
 *   SampleVoxelSpace   src/kernel.cpp:96-126
 *   RNG_Sample         src/kernel.cpp:55-69
 */
#include "kernel.cpp"

extern "C" float ref_sample_voxel_space(const float p[3], const float *brick, const float ce[4], unsigned lvoxc) {
    float4 P(p[0], p[1], p[2], 0.0f);
    float4 CE(ce[0], ce[1], ce[2], ce[3]);
    return SampleVoxelSpace(P, const_cast<float *>(brick), CE, lvoxc);
}

/* Draws n numbers from lane 0..3 of one reference RNG state seeded with s[16]. */
extern "C" void ref_rng_draw(const unsigned s[16], unsigned n, float *out4) {
    sint4 st;
    for (int i = 0; i < 4; ++i)
        st.v[i].v = _mm_set_epi32((int)s[4 * i + 3], (int)s[4 * i + 2], (int)s[4 * i + 1], (int)s[4 * i + 0]);
    for (unsigned k = 0; k < n; ++k) {
        __m128 r = RNG_Sample(&st);
        _mm_storeu_ps(out4 + 4 * k, r);
    }
}
