// Intersection handler used by the tests: each AABB holds the sphere inscribed in its x extent.
__device__ lam_aabb_intersection intersect(const lam_ray_intersection& i) {
    lam_aabb_intersection r;
    r.hit = 0u;
    r.t = 0.0f;
    for (int k = 0; k < 3; ++k) r.normal[k] = r.tangent[k] = 0.0f;
    const float rad = 0.5f * (i.aabb_max[0] - i.aabb_min[0]);
    float oc[3], d[3];
    for (int k = 0; k < 3; ++k) {
        oc[k] = i.object_origin[k] - 0.5f * (i.aabb_min[k] + i.aabb_max[k]);
        d[k] = i.object_direction[k];
    }
    const float a = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const float b = oc[0] * d[0] + oc[1] * d[1] + oc[2] * d[2];
    const float c = oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2] - rad * rad;
    const float disc = b * b - a * c;
    if (!(disc >= 0.0f) || !(a > 0.0f)) return r;
    const float s = sqrtf(disc);
    float t = (-b - s) / a;
    if (!(t > i.tmin)) t = (-b + s) / a;
    if (!(t > i.tmin)) return r;
    r.hit = 1u;
    r.t = t;
    for (int k = 0; k < 3; ++k) r.normal[k] = (oc[k] + t * d[k]) / rad;
    r.tangent[0] = -r.normal[2];
    r.tangent[1] = 0.0f;
    r.tangent[2] = r.normal[0];
    return r;
}
