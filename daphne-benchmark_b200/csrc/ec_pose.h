// Box yaw of a cluster's bounding box (host code, ec_pose.cpp).
#pragma once

namespace ec {
// xyz: the cluster's n points (3 floats each); min_x / min_y: their smallest
// x and y.  Writes the z and w of the yaw quaternion (x = y = 0).
void box_yaw(const float *xyz, int n, float min_x, float min_y, double *qz, double *qw);

// Many clusters at once, spread over up to kYawThreads host threads.
constexpr int kYawThreads = 8;
struct YawJob {
    const float *xyz;
    int n;
    float min_x, min_y;
    double *qz, *qw;
};
void box_yaws(const YawJob *jobs, int count);
}  // namespace ec
