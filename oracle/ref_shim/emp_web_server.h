// Project-written stand-in that shadows the reference's include/emp_web_server.h
// (microhttpd, only used when WEBSERVER is defined, which oracle/_ref never does).
#ifndef EMP_WEB_SERVER_H
#define EMP_WEB_SERVER_H
namespace edge_matching_puzzle {
class emp_web_server;
}
#endif
