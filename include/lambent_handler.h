/* lambent_handler.h - the types an intersection handler sees (RayTracer::set_intersection_handler,
 * src/lib.rs:291-295; IntersectionHandler, src/low_level.rs:115-147).  Plain C with built-in types
 * only: the same text is handed to the runtime compiler together with the handler's source. */
#ifndef LAMBENT_HANDLER_H
#define LAMBENT_HANDLER_H

#define LAM_INTERSECTION_AABB 2u

/* RayIntersection of the candidate (the WGSL ray-query candidate fields, general.wesl:1058), plus
 * the ray itself and the candidate's box, which a handler needs and the reference's cannot see. */
typedef struct lam_ray_intersection {
    unsigned int kind;                  /* LAM_INTERSECTION_AABB */
    float t;                            /* closest committed distance so far (tmax when none) */
    unsigned int instance_custom_data;
    unsigned int instance_index;
    unsigned int sbt_record_offset;     /* 0 */
    unsigned int geometry_index;        /* 0 */
    unsigned int primitive_index;
    float barycentrics[2];              /* 0 for AABB candidates */
    unsigned int front_face;            /* 0 for AABB candidates */
    float object_to_world[12];          /* 3x4 row-major */
    float world_to_object[12];
    float world_origin[3], world_direction[3];
    float object_origin[3], object_direction[3];
    float tmin;
    float aabb_min[3], aabb_max[3];     /* the candidate's box in object space */
} lam_ray_intersection;

/* AABBIntersection (src/intersection.wesl): a hit at ray parameter t commits when tmin < t and it
 * is closer than the committed hit; normal and tangent become the hit's. */
typedef struct lam_aabb_intersection {
    unsigned int hit;
    float normal[3];
    float tangent[3];
    float t;
} lam_aabb_intersection;

#endif /* LAMBENT_HANDLER_H */
