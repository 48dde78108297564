// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,12,1,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,12,1,12>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1920,120,12,10,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1920,120,12,10,16>(const PassDesc);
extern const StaticPlan kPlans_f64_3[];
extern const int kPlansCount_f64_3;
const StaticPlan kPlans_f64_3[] = {
  {4, 1, 1, {4}, 1024, (const void*)&axis_pass_static<double,true,1024,4,1,4>, (const void*)&axis_pass_static<double,false,1024,4,1,4>, nullptr, nullptr, 512, 0},
  {12, 1, 1, {12}, 512, (const void*)&axis_pass_static<double,true,512,12,1,12>, (const void*)&axis_pass_static<double,false,512,12,1,12>, (const void*)&axis_pass_pipe<double,512,false,8,12,1,12>, (const void*)&axis_pass_pipe<double,512,true,0,12,1,12>, 512, 8},
  {25, 5, 2, {5,5}, 1024, (const void*)&axis_pass_static<double,true,1024,25,5,5,5>, (const void*)&axis_pass_static<double,false,1024,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,false,8,25,5,5,5>, (const void*)&axis_pass_pipe<double,512,true,0,25,5,5,5>, 512, 8},
  {45, 3, 2, {15,3}, 512, (const void*)&axis_pass_static<double,true,512,45,3,15,3>, (const void*)&axis_pass_static<double,false,512,45,3,15,3>, (const void*)&axis_pass_pipe<double,512,false,8,45,3,15,3>, (const void*)&axis_pass_pipe<double,512,true,0,45,3,15,3>, 512, 8},
  {72, 6, 2, {12,6}, 512, (const void*)&axis_pass_static<double,true,512,72,6,12,6>, (const void*)&axis_pass_static<double,false,512,72,6,12,6>, (const void*)&axis_pass_pipe<double,512,false,8,72,6,12,6>, (const void*)&axis_pass_pipe<double,512,true,0,72,6,12,6>, 512, 8},
  {100, 10, 2, {10,10}, 512, (const void*)&axis_pass_static<double,true,512,100,10,10,10>, (const void*)&axis_pass_static<double,false,512,100,10,10,10>, (const void*)&axis_pass_pipe<double,512,false,8,100,10,10,10>, (const void*)&axis_pass_pipe<double,512,true,0,100,10,10,10>, 512, 8},
  {144, 12, 2, {12,12}, 512, (const void*)&axis_pass_static<double,true,512,144,12,12,12>, (const void*)&axis_pass_static<double,false,512,144,12,12,12>, (const void*)&axis_pass_pipe<double,512,false,8,144,12,12,12>, (const void*)&axis_pass_pipe<double,512,true,0,144,12,12,12>, 512, 8},
  {200, 25, 3, {5,5,8}, 512, (const void*)&axis_pass_static<double,true,512,200,25,5,5,8>, (const void*)&axis_pass_static<double,false,512,200,25,5,5,8>, (const void*)&axis_pass_pipe<double,512,false,8,200,25,5,5,8>, (const void*)&axis_pass_pipe<double,512,true,0,200,25,5,5,8>, 512, 8},
  {256, 16, 2, {16,16}, 512, (const void*)&axis_pass_static<double,true,512,256,16,16,16>, (const void*)&axis_pass_static<double,false,512,256,16,16,16>, (const void*)&axis_pass_pipe<double,512,false,8,256,16,16,16>, (const void*)&axis_pass_pipe<double,512,true,0,256,16,16,16>, 512, 8},
  {360, 36, 3, {10,6,6}, 512, (const void*)&axis_pass_static<double,true,512,360,36,10,6,6>, (const void*)&axis_pass_static<double,false,512,360,36,10,6,6>, (const void*)&axis_pass_pipe<double,512,false,8,360,36,10,6,6>, (const void*)&axis_pass_pipe<double,512,true,0,360,36,10,6,6>, 512, 8},
  {450, 30, 3, {15,6,5}, 512, (const void*)&axis_pass_static<double,true,512,450,30,15,6,5>, (const void*)&axis_pass_static<double,false,512,450,30,15,6,5>, (const void*)&axis_pass_pipe<double,512,false,8,450,30,15,6,5>, (const void*)&axis_pass_pipe<double,512,true,0,450,30,15,6,5>, 512, 8},
  {576, 48, 3, {12,6,8}, 512, (const void*)&axis_pass_static<double,true,512,576,48,12,6,8>, (const void*)&axis_pass_static<double,false,512,576,48,12,6,8>, nullptr, nullptr, 512, 0},
  {720, 60, 3, {12,10,6}, 512, (const void*)&axis_pass_static<double,true,512,720,60,12,10,6>, (const void*)&axis_pass_static<double,false,512,720,60,12,10,6>, nullptr, nullptr, 512, 0},
  {864, 72, 3, {12,12,6}, 512, (const void*)&axis_pass_static<double,true,512,864,72,12,12,6>, (const void*)&axis_pass_static<double,false,512,864,72,12,12,6>, nullptr, nullptr, 512, 0},
  {1080, 72, 3, {15,12,6}, 512, (const void*)&axis_pass_static<double,true,512,1080,72,15,12,6>, (const void*)&axis_pass_static<double,false,512,1080,72,15,12,6>, nullptr, nullptr, 512, 0},
  {1280, 80, 3, {10,16,8}, 512, (const void*)&axis_pass_static<double,true,512,1280,80,10,16,8>, (const void*)&axis_pass_static<double,false,512,1280,80,10,16,8>, nullptr, nullptr, 512, 0},
  {1536, 96, 3, {12,16,8}, 512, (const void*)&axis_pass_static<double,true,512,1536,96,12,16,8>, (const void*)&axis_pass_static<double,false,512,1536,96,12,16,8>, nullptr, nullptr, 512, 0},
  {1920, 120, 3, {12,10,16}, 512, (const void*)&axis_pass_static<double,true,512,1920,120,12,10,16>, (const void*)&axis_pass_static<double,false,512,1920,120,12,10,16>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_3 = 18;
}  // namespace dfft
