// Generated by gen_crmath_tables.py -- do not edit.
// Double-double (hi, lo) splits, exact hex-float literals.
#pragma once

namespace bgt {
namespace cr {

#ifdef __CUDACC__
__constant__ double SIN_C_dev[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.5555555555555p-3, -0x1.5555555555555p-57},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {-0x1.434d2e783f5bcp-113, -0x1.0b87b91be9affp-167},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
};
#endif
static const double SIN_C_host[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.5555555555555p-3, -0x1.5555555555555p-57},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {-0x1.434d2e783f5bcp-113, -0x1.0b87b91be9affp-167},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
};
#ifdef __CUDA_ARCH__
#define SIN_C SIN_C_dev
#else
#define SIN_C SIN_C_host
#endif
#ifdef __CUDACC__
__constant__ double COS_C_dev[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {-0x1.3932c5047d60ep-108, -0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
};
#endif
static const double COS_C_host[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {-0x1.3932c5047d60ep-108, -0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
};
#ifdef __CUDA_ARCH__
#define COS_C COS_C_dev
#else
#define COS_C COS_C_host
#endif
#ifdef __CUDACC__
__constant__ double SINH_C_dev[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {0x1.434d2e783f5bcp-113, 0x1.0b87b91be9affp-167},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
};
#endif
static const double SINH_C_host[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {0x1.434d2e783f5bcp-113, 0x1.0b87b91be9affp-167},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
};
#ifdef __CUDA_ARCH__
#define SINH_C SINH_C_dev
#else
#define SINH_C SINH_C_host
#endif
#ifdef __CUDACC__
__constant__ double COSH_C_dev[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {0x1.3932c5047d60ep-108, 0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
};
#endif
static const double COSH_C_host[17][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {0x1.3932c5047d60ep-108, 0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
};
#ifdef __CUDA_ARCH__
#define COSH_C COSH_C_dev
#else
#define COSH_C COSH_C_host
#endif
#ifdef __CUDACC__
__constant__ double EXP_C_dev[41][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {0x1.3932c5047d60ep-108, 0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-113, 0x1.0b87b91be9affp-167},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
    {0x1.2710231c0fd7ap-128, 0x1.3f8a2b4af9d6bp-184},
    {0x1.0dc59c716d91fp-133, 0x1.419e3fad3f031p-188},
    {0x1.df983290c2ca9p-139, 0x1.5835c6895393bp-194},
    {0x1.9ec8d1c94e85bp-144, -0x1.670e9d4784ec6p-201},
    {0x1.5d4acb9c0c3abp-149, -0x1.6ec2c8f5b13b2p-205},
    {0x1.1e99449a4bacep-154, -0x1.fefbb89514b3cp-210},
    {0x1.ca8ed42a12ae3p-160, 0x1.a07244abad2abp-224},
};
#endif
static const double EXP_C_host[41][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p+0, 0.0},
    {0x1.0000000000000p-1, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {0x1.6c16c16c16c17p-10, -0x1.f49f49f49f49fp-65},
    {0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {0x1.27e4fb7789f5cp-22, 0x1.cbbc05b4fa99ap-76},
    {0x1.ae64567f544e4p-26, -0x1.c062e06d1f209p-80},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {0x1.93974a8c07c9dp-37, 0x1.05d6f8a2efd1fp-92},
    {0x1.ae7f3e733b81fp-41, 0x1.1d8656b0ee8cbp-97},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {0x1.6827863b97d97p-53, 0x1.eec01221a8b0bp-107},
    {0x1.2f49b46814157p-57, 0x1.2650f61dbdcb4p-112},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {0x1.0ce396db7f853p-70, -0x1.aebcdbd20331cp-124},
    {0x1.761b41316381ap-75, -0x1.3423c7d91404fp-130},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {0x1.88e85fc6a4e5ap-89, -0x1.71c37ebd16540p-143},
    {0x1.d1ab1c2dccea3p-94, 0x1.054d0c78aea14p-149},
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153},
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157},
    {0x1.3932c5047d60ep-108, 0x1.832b7b530a627p-162},
    {0x1.434d2e783f5bcp-113, 0x1.0b87b91be9affp-167},
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172},
    {0x1.3981254dd0d52p-123, -0x1.2b1f4c8015a2fp-177},
    {0x1.2710231c0fd7ap-128, 0x1.3f8a2b4af9d6bp-184},
    {0x1.0dc59c716d91fp-133, 0x1.419e3fad3f031p-188},
    {0x1.df983290c2ca9p-139, 0x1.5835c6895393bp-194},
    {0x1.9ec8d1c94e85bp-144, -0x1.670e9d4784ec6p-201},
    {0x1.5d4acb9c0c3abp-149, -0x1.6ec2c8f5b13b2p-205},
    {0x1.1e99449a4bacep-154, -0x1.fefbb89514b3cp-210},
    {0x1.ca8ed42a12ae3p-160, 0x1.a07244abad2abp-224},
};
#ifdef __CUDA_ARCH__
#define EXP_C EXP_C_dev
#else
#define EXP_C EXP_C_host
#endif
#ifdef __CUDACC__
__constant__ double ASIN_C_dev[40][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.3333333333333p-4, 0x1.999999999999ap-59},
    {0x1.6db6db6db6db7p-5, -0x1.2492492492492p-60},
    {0x1.f1c71c71c71c7p-6, 0x1.c71c71c71c71cp-62},
    {0x1.6e8ba2e8ba2e9p-6, -0x1.1745d1745d174p-60},
    {0x1.1c4ec4ec4ec4fp-6, -0x1.d89d89d89d89ep-61},
    {0x1.c99999999999ap-7, -0x1.999999999999ap-61},
    {0x1.7a87878787878p-7, 0x1.e1e1e1e1e1e1ep-61},
    {0x1.3fde50d79435ep-7, 0x1.435e50d79435ep-61},
    {0x1.12ef3cf3cf3cfp-7, 0x1.e79e79e79e79ep-62},
    {0x1.df3bd37a6f4dfp-8, -0x1.90b21642c8591p-62},
    {0x1.a6863d70a3d71p-8, -0x1.70a3d70a3d70ap-62},
    {0x1.782dda12f684cp-8, -0x1.2f684bda12f68p-63},
    {0x1.51ba308d3dcb1p-8, -0x1.cb08d3dcb08d4p-62},
    {0x1.31683bdef7bdfp-8, -0x1.0842108421084p-65},
    {0x1.15ee9d45d1746p-8, -0x1.745d1745d1746p-63},
    {0x1.fcaf8fb6db6dbp-9, 0x1.b6db6db6db6dbp-63},
    {0x1.d3d2a8e0dd67dp-9, -0x1.d67c8a60dd67dp-63},
    {0x1.b026f57b13b14p-9, -0x1.3b13b13b13b14p-63},
    {0x1.90cb77f60c7cep-9, 0x1.8f9c18f9c18fap-66},
    {0x1.750de64d7d05fp-9, 0x1.05f417d05f418p-63},
    {0x1.5c5f56efaaaabp-9, -0x1.5555555555555p-63},
    {0x1.464c0950f7d47p-9, -0x1.882b931057262p-64},
    {0x1.3275586c5f2f0p-9, 0x1.4e5e0a72f0539p-63},
    {0x1.208d3570ae5a6p-9, -0x1.6969696969697p-63},
    {0x1.1052bc5fa960ap-9, -0x1.5bc609a90e7d9p-63},
    {0x1.018f963c229bfp-9, -0x1.4f2094f2094f2p-64},
    {0x1.e82be60d9127ep-10, -0x1.f7047dc11f704p-65},
    {0x1.cf7dea5b6e830p-10, -0x1.15b1e5f75270dp-64},
    {0x1.b8d2e5667ce6cp-10, 0x1.0c9714fbcda3bp-66},
    {0x1.a3f1ef82137eep-10, 0x1.c71c71c71c71cp-65},
    {0x1.90a9f747db95dp-10, -0x1.6a56a56a56a57p-65},
    {0x1.7ed079ed4c037p-10, -0x1.03d226357e16fp-66},
    {0x1.6e40790442038p-10, 0x1.a6f4de9bd37a7p-67},
    {0x1.5ed9a0bd901b6p-10, -0x1.040e6c2b4481dp-64},
    {0x1.507f94c2470bdp-10, 0x1.56070381c0e07p-65},
    {0x1.43195bf54e5d7p-10, -0x1.b9e4b17e4b17ep-64},
    {0x1.3690e51f04536p-10, 0x1.9d9745d1745d1p-64},
    {0x1.2ad29fcd49d54p-10, 0x1.82fbf309b8b57p-64},
};
#endif
static const double ASIN_C_host[40][2] = {
    {0x1.0000000000000p+0, 0.0},
    {0x1.5555555555555p-3, 0x1.5555555555555p-57},
    {0x1.3333333333333p-4, 0x1.999999999999ap-59},
    {0x1.6db6db6db6db7p-5, -0x1.2492492492492p-60},
    {0x1.f1c71c71c71c7p-6, 0x1.c71c71c71c71cp-62},
    {0x1.6e8ba2e8ba2e9p-6, -0x1.1745d1745d174p-60},
    {0x1.1c4ec4ec4ec4fp-6, -0x1.d89d89d89d89ep-61},
    {0x1.c99999999999ap-7, -0x1.999999999999ap-61},
    {0x1.7a87878787878p-7, 0x1.e1e1e1e1e1e1ep-61},
    {0x1.3fde50d79435ep-7, 0x1.435e50d79435ep-61},
    {0x1.12ef3cf3cf3cfp-7, 0x1.e79e79e79e79ep-62},
    {0x1.df3bd37a6f4dfp-8, -0x1.90b21642c8591p-62},
    {0x1.a6863d70a3d71p-8, -0x1.70a3d70a3d70ap-62},
    {0x1.782dda12f684cp-8, -0x1.2f684bda12f68p-63},
    {0x1.51ba308d3dcb1p-8, -0x1.cb08d3dcb08d4p-62},
    {0x1.31683bdef7bdfp-8, -0x1.0842108421084p-65},
    {0x1.15ee9d45d1746p-8, -0x1.745d1745d1746p-63},
    {0x1.fcaf8fb6db6dbp-9, 0x1.b6db6db6db6dbp-63},
    {0x1.d3d2a8e0dd67dp-9, -0x1.d67c8a60dd67dp-63},
    {0x1.b026f57b13b14p-9, -0x1.3b13b13b13b14p-63},
    {0x1.90cb77f60c7cep-9, 0x1.8f9c18f9c18fap-66},
    {0x1.750de64d7d05fp-9, 0x1.05f417d05f418p-63},
    {0x1.5c5f56efaaaabp-9, -0x1.5555555555555p-63},
    {0x1.464c0950f7d47p-9, -0x1.882b931057262p-64},
    {0x1.3275586c5f2f0p-9, 0x1.4e5e0a72f0539p-63},
    {0x1.208d3570ae5a6p-9, -0x1.6969696969697p-63},
    {0x1.1052bc5fa960ap-9, -0x1.5bc609a90e7d9p-63},
    {0x1.018f963c229bfp-9, -0x1.4f2094f2094f2p-64},
    {0x1.e82be60d9127ep-10, -0x1.f7047dc11f704p-65},
    {0x1.cf7dea5b6e830p-10, -0x1.15b1e5f75270dp-64},
    {0x1.b8d2e5667ce6cp-10, 0x1.0c9714fbcda3bp-66},
    {0x1.a3f1ef82137eep-10, 0x1.c71c71c71c71cp-65},
    {0x1.90a9f747db95dp-10, -0x1.6a56a56a56a57p-65},
    {0x1.7ed079ed4c037p-10, -0x1.03d226357e16fp-66},
    {0x1.6e40790442038p-10, 0x1.a6f4de9bd37a7p-67},
    {0x1.5ed9a0bd901b6p-10, -0x1.040e6c2b4481dp-64},
    {0x1.507f94c2470bdp-10, 0x1.56070381c0e07p-65},
    {0x1.43195bf54e5d7p-10, -0x1.b9e4b17e4b17ep-64},
    {0x1.3690e51f04536p-10, 0x1.9d9745d1745d1p-64},
    {0x1.2ad29fcd49d54p-10, 0x1.82fbf309b8b57p-64},
};
#ifdef __CUDA_ARCH__
#define ASIN_C ASIN_C_dev
#else
#define ASIN_C ASIN_C_host
#endif
#ifdef __CUDACC__
__constant__ double ATAN_C_dev[40][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.5555555555555p-2, -0x1.5555555555555p-56},
    {0x1.999999999999ap-3, -0x1.999999999999ap-57},
    {-0x1.2492492492492p-3, -0x1.2492492492492p-57},
    {0x1.c71c71c71c71cp-4, 0x1.c71c71c71c71cp-58},
    {-0x1.745d1745d1746p-4, 0x1.745d1745d1746p-59},
    {0x1.3b13b13b13b14p-4, -0x1.3b13b13b13b14p-58},
    {-0x1.1111111111111p-4, -0x1.1111111111111p-60},
    {0x1.e1e1e1e1e1e1ep-5, 0x1.e1e1e1e1e1e1ep-61},
    {-0x1.af286bca1af28p-5, -0x1.af286bca1af28p-59},
    {0x1.8618618618618p-5, 0x1.8618618618618p-59},
    {-0x1.642c8590b2164p-5, -0x1.642c8590b2164p-60},
    {0x1.47ae147ae147bp-5, -0x1.eb851eb851eb8p-61},
    {-0x1.2f684bda12f68p-5, -0x1.2f684bda12f68p-59},
    {0x1.1a7b9611a7b96p-5, 0x1.1a7b9611a7b96p-61},
    {-0x1.0842108421084p-5, -0x1.0842108421084p-60},
    {0x1.f07c1f07c1f08p-6, -0x1.f07c1f07c1f08p-61},
    {-0x1.d41d41d41d41dp-6, -0x1.0750750750750p-60},
    {0x1.bacf914c1bad0p-6, -0x1.bacf914c1bad0p-60},
    {-0x1.a41a41a41a41ap-6, -0x1.0690690690690p-60},
    {0x1.8f9c18f9c18fap-6, -0x1.f3831f3831f38p-61},
    {-0x1.7d05f417d05f4p-6, -0x1.7d05f417d05f4p-62},
    {0x1.6c16c16c16c17p-6, -0x1.f49f49f49f49fp-61},
    {-0x1.5c9882b931057p-6, -0x1.310572620ae4cp-61},
    {0x1.4e5e0a72f0539p-6, 0x1.e0a72f0539783p-60},
    {-0x1.4141414141414p-6, -0x1.4141414141414p-62},
    {0x1.3521cfb2b78c1p-6, 0x1.a90e7d95bc60ap-61},
    {-0x1.29e4129e4129ep-6, -0x1.04a7904a7904ap-60},
    {0x1.1f7047dc11f70p-6, 0x1.1f7047dc11f70p-60},
    {-0x1.15b1e5f75270dp-6, -0x1.15b1e5f75270dp-64},
    {0x1.0c9714fbcda3bp-6, -0x1.f79b47582192ep-61},
    {-0x1.0410410410410p-6, -0x1.0410410410410p-60},
    {0x1.f81f81f81f820p-7, -0x1.f81f81f81f820p-61},
    {-0x1.e9131abf0b767p-7, -0x1.503d226357e17p-62},
    {0x1.dae6076b981dbp-7, -0x1.9f89467e251a0p-63},
    {-0x1.cd85689039b0bp-7, 0x1.76fc64f52edf9p-62},
    {0x1.c0e070381c0e0p-7, 0x1.c0e070381c0e0p-61},
    {-0x1.b4e81b4e81b4fp-7, 0x1.f92c5f92c5f93p-61},
    {0x1.a98ef606a63bep-7, -0x1.f959c427e5671p-61},
    {-0x1.9ec8e951033d9p-7, -0x1.d2a2067b23a54p-63},
};
#endif
static const double ATAN_C_host[40][2] = {
    {0x1.0000000000000p+0, 0.0},
    {-0x1.5555555555555p-2, -0x1.5555555555555p-56},
    {0x1.999999999999ap-3, -0x1.999999999999ap-57},
    {-0x1.2492492492492p-3, -0x1.2492492492492p-57},
    {0x1.c71c71c71c71cp-4, 0x1.c71c71c71c71cp-58},
    {-0x1.745d1745d1746p-4, 0x1.745d1745d1746p-59},
    {0x1.3b13b13b13b14p-4, -0x1.3b13b13b13b14p-58},
    {-0x1.1111111111111p-4, -0x1.1111111111111p-60},
    {0x1.e1e1e1e1e1e1ep-5, 0x1.e1e1e1e1e1e1ep-61},
    {-0x1.af286bca1af28p-5, -0x1.af286bca1af28p-59},
    {0x1.8618618618618p-5, 0x1.8618618618618p-59},
    {-0x1.642c8590b2164p-5, -0x1.642c8590b2164p-60},
    {0x1.47ae147ae147bp-5, -0x1.eb851eb851eb8p-61},
    {-0x1.2f684bda12f68p-5, -0x1.2f684bda12f68p-59},
    {0x1.1a7b9611a7b96p-5, 0x1.1a7b9611a7b96p-61},
    {-0x1.0842108421084p-5, -0x1.0842108421084p-60},
    {0x1.f07c1f07c1f08p-6, -0x1.f07c1f07c1f08p-61},
    {-0x1.d41d41d41d41dp-6, -0x1.0750750750750p-60},
    {0x1.bacf914c1bad0p-6, -0x1.bacf914c1bad0p-60},
    {-0x1.a41a41a41a41ap-6, -0x1.0690690690690p-60},
    {0x1.8f9c18f9c18fap-6, -0x1.f3831f3831f38p-61},
    {-0x1.7d05f417d05f4p-6, -0x1.7d05f417d05f4p-62},
    {0x1.6c16c16c16c17p-6, -0x1.f49f49f49f49fp-61},
    {-0x1.5c9882b931057p-6, -0x1.310572620ae4cp-61},
    {0x1.4e5e0a72f0539p-6, 0x1.e0a72f0539783p-60},
    {-0x1.4141414141414p-6, -0x1.4141414141414p-62},
    {0x1.3521cfb2b78c1p-6, 0x1.a90e7d95bc60ap-61},
    {-0x1.29e4129e4129ep-6, -0x1.04a7904a7904ap-60},
    {0x1.1f7047dc11f70p-6, 0x1.1f7047dc11f70p-60},
    {-0x1.15b1e5f75270dp-6, -0x1.15b1e5f75270dp-64},
    {0x1.0c9714fbcda3bp-6, -0x1.f79b47582192ep-61},
    {-0x1.0410410410410p-6, -0x1.0410410410410p-60},
    {0x1.f81f81f81f820p-7, -0x1.f81f81f81f820p-61},
    {-0x1.e9131abf0b767p-7, -0x1.503d226357e17p-62},
    {0x1.dae6076b981dbp-7, -0x1.9f89467e251a0p-63},
    {-0x1.cd85689039b0bp-7, 0x1.76fc64f52edf9p-62},
    {0x1.c0e070381c0e0p-7, 0x1.c0e070381c0e0p-61},
    {-0x1.b4e81b4e81b4fp-7, 0x1.f92c5f92c5f93p-61},
    {0x1.a98ef606a63bep-7, -0x1.f959c427e5671p-61},
    {-0x1.9ec8e951033d9p-7, -0x1.d2a2067b23a54p-63},
};
#ifdef __CUDA_ARCH__
#define ATAN_C ATAN_C_dev
#else
#define ATAN_C ATAN_C_host
#endif
#define BGT_CR_PI_HI 0x1.921fb54442d18p+1
#define BGT_CR_PI_LO 0x1.1a62633145c07p-53
#define BGT_CR_PIO2_HI 0x1.921fb54442d18p+0
#define BGT_CR_PIO2_LO 0x1.1a62633145c07p-54
#define BGT_CR_TWO_OVER_PI 0x1.45f306dc9c883p-1
// pi/2 = CW1 + CW2 + CW3; CW1 and CW2 carry 33 significant bits
#define BGT_CR_PIO2_CW1 0x1.921fb54400000p+0
#define BGT_CR_PIO2_CW2 0x1.0b4611a600000p-34
#define BGT_CR_PIO2_CW3 0x1.3198a2e037073p-69

}  // namespace cr
}  // namespace bgt

